"""The oracle's assembly and solve against the reference's own code.

oracle/_ref/libdare_ref.so is the reference's DDT / Gradient / Divergence /
TVD / MatrixBlock code (Grid/Cartesian, Equations, Data, MatrixSystem),
compiled from its own headers against single-rank stand-ins for MPI, Kokkos
and Tpetra, run through the per-cell loop of Trilinos<SC>::BuildNew
(MatrixSystem/Trilinos.inl:285-385) with the functor of the reference's
drivers (test/Verification/counter_diffusion1D.cpp:107-148).  The C
restatement in oracle/dare_oracle.c must reproduce it bit for bit: row
pointers, sorted columns, coefficients, right-hand side and initial guess, on
seeded random grids in one to three dimensions with every limiter, every time
scheme the reference compiles, scalar and face diffusivities and Dirichlet /
Neumann faces.  The same library holds the reference's BiCGStab2
(MatrixSystem/BiCGStab2.h, .inl) over a CSR operator and vectors that restate
Tpetra's update / dot / norm2 / apply, with Ifpack2's Jacobi on the right; the
oracle's solve (one thread, so its sums run in index order) must give the same
iterates bit for bit: iteration count, convergence flag and solution.  The
library is built where the reference's sources are present
(``make -C oracle ref``).
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (the reference's sources are absent)")

LIMS = [("CDS", O.LIM_CDS), ("UPWIND", O.LIM_UPWIND), ("VANALBADA", O.LIM_VANALBADA), ("MINMOD", O.LIM_MINMOD),
        ("VANLEER", O.LIM_VANLEER)]
SCHEMES = [("EULER_BACKWARD", O.SCHEME_EULER_BACKWARD), ("EULER_FORWARD", O.SCHEME_EULER_FORWARD),
           ("CRANK_NICHOLSON", O.SCHEME_CRANK_NICHOLSON), ("ADAMS_BASHFORT", O.SCHEME_ADAMS_BASHFORTH)]


def face_arrays(rng, dim, n, lo=1e-5, hi=1e-2):
    nn = [n[q] if q < dim else 1 for q in range(3)]
    out = []
    for q in range(dim):
        shape = list(nn)
        shape[q] += 1
        out.append(np.exp(rng.uniform(np.log(lo), np.log(hi), size=int(np.prod(shape)))))
    return out


def field(rng, og, kind):
    size = int(np.prod(O.ghosted_shape(og)))
    if kind == "normal":
        phi = rng.normal(size=size)
    elif kind == "decades":     # values over twelve decades with random signs
        phi = rng.choice([-1.0, 1.0], size=size) * 10.0 ** rng.uniform(-6, 6, size=size)
    else:                       # plateaus: equal neighbours give r = 0/0 and r = x/0 in the limiters
        phi = rng.integers(0, 3, size=size).astype(np.float64)
    O.exchange_halo(og, phi)
    return phi


def compare(dim, n, periodic, rng, *, dt, D=None, face_D=None, vel=None, lim=("VANLEER", O.LIM_VANLEER),
            scheme=("EULER_BACKWARD", O.SCHEME_EULER_BACKWARD), bc=None, kind="normal"):
    size = [1.0 + 0.5 * q for q in range(dim)]
    og = O.make_grid(dim, n, size, 2, periodic)
    phi, old = field(rng, og, kind), field(rng, og, "normal")
    ofd = None if face_D is None else list(face_D) + [None] * (3 - len(face_D))
    desc = O.AssemblyDesc(og, dt=dt, D=D, face_D=ofd, vel=vel, limiter=lim[1], bc=bc, scheme=scheme[1])
    diag, rhs, mask = O.assemble(desc, phi, old)
    rp, cols, vals = O.export_csr(og, diag, mask)
    x0 = O.field_to_vector(og, phi)
    rrp, rcols, rvals, rrhs, rx0 = R.assemble(dim, n, size, periodic, phi, old, dt=dt, D=D, face_D=face_D, vel=vel,
                                              limiter=lim[0], scheme=scheme[0], bc=bc)
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(cols, rcols)
    # bit for bit, NaN where the reference gives NaN
    assert np.array_equal(vals.view(np.int64), rvals.view(np.int64)) or np.array_equal(vals, rvals, equal_nan=True), \
        np.max(np.abs(vals - rvals))
    assert np.array_equal(rhs, rrhs, equal_nan=True), np.nanmax(np.abs(rhs - rrhs))
    np.testing.assert_array_equal(x0, rx0)


def random_bc(rng, dim, periodic):
    bc = {}
    for q in range(dim):
        if periodic[q]:
            continue
        for side in range(2):
            bc[2 * q + 1 + side] = (int(rng.integers(1, 3)), float(rng.uniform(-1, 1)))
    return bc


@pytest.mark.parametrize("seed", range(24))
def test_random_configurations(seed):
    rng = np.random.default_rng(1000 + seed)
    dim = 1 + seed % 3
    periodic = tuple(int(rng.integers(0, 2)) for _ in range(dim))
    n = tuple(int(rng.integers(3, 9 if dim == 3 else 13)) for _ in range(dim))
    lim = LIMS[seed % len(LIMS)]
    scheme = SCHEMES[(seed // 3) % len(SCHEMES)]
    dt = 0.0 if seed % 7 == 6 else float(10.0 ** rng.uniform(-3, -1))
    vel = None if seed % 5 == 4 else tuple(float(rng.choice([-1, 0, 1]) * rng.uniform(0.05, 1.0)) for _ in range(dim))
    kw = {}
    if seed % 4 == 3:
        kw["face_D"] = face_arrays(rng, dim, n)
    elif seed % 4 != 2:
        kw["D"] = float(10.0 ** rng.uniform(-5, -2))
    kind = ["normal", "decades", "plateaus"][seed % 3]
    compare(dim, n, periodic, rng, dt=dt, vel=vel, lim=lim, scheme=scheme, bc=random_bc(rng, dim, periodic),
            kind=kind, **kw)


@pytest.mark.parametrize("lim", LIMS, ids=[l[0] for l in LIMS])
@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_tvd_every_limiter_both_directions(lim, sign):
    """Convection-diffusion on a periodic 3-D grid (the headline operator with
    a constant velocity) and on a bounded one, every limiter, both flow
    directions."""
    rng = np.random.default_rng(7)
    vel = (sign * 0.4, -sign * 0.25, sign * 0.1)
    compare(3, (6, 5, 7), (1, 1, 1), rng, dt=1.5e-2, D=1e-4, vel=vel, lim=lim)
    compare(3, (6, 5, 7), (0, 1, 0), rng, dt=1.5e-2, D=1e-4, vel=vel, lim=lim,
            bc={1: (1, 1.0), 2: (1, 0.0), 5: (2, 0.0), 6: (2, 0.0)})


def test_counter_diffusion_and_config0_operators():
    """The counter-diffusion driver's operator (1-D, Dirichlet at one end and
    Neumann at the other) and the Gaussian-diffusion workload's operator on a
    16^3 grid (Dirichlet 1 / 0 on x, Neumann elsewhere)."""
    rng = np.random.default_rng(3)
    compare(1, (10,), (0,), rng, dt=1e-3, D=1.0, bc={1: (1, 1.0), 2: (2, 0.0)})
    compare(1, (10,), (0,), rng, dt=1e-3, D=1.0, bc={1: (2, 0.0), 2: (1, 1.0)})
    bc = {1: (1, 1.0), 2: (1, 0.0), 3: (2, 0.0), 4: (2, 0.0), 5: (2, 0.0), 6: (2, 0.0)}
    compare(3, (16, 16, 16), (0, 0, 0), rng, dt=1e-2, D=1e-3, bc=bc)


def test_heterogeneous_face_diffusivity_3d():
    """Face diffusivities over three decades with TVD convection (the
    operator of the heterogeneous workload), periodic and bounded."""
    rng = np.random.default_rng(11)
    n = (7, 6, 8)
    compare(3, n, (1, 1, 1), rng, dt=3.8e-3, face_D=face_arrays(rng, 3, n, 1e-5, 1e-2), vel=(0.2, 0.1, -0.3))
    compare(3, n, (0, 0, 1), rng, dt=3.8e-3, face_D=face_arrays(rng, 3, n, 1e-5, 1e-2), vel=(-0.2, 0.1, 0.3),
            bc={1: (1, 0.2), 2: (2, 0.0), 3: (1, 0.7), 4: (1, -0.1)})


def solve_both(rp, cols, vals, rhs, x0, tol, max_it, jacobi):
    threads = O.num_threads()
    O.set_threads(1)   # one OpenMP thread for both libraries: sums in index order
    try:
        xo, info = O.bicgstab2(rp, cols, vals, rhs, x0, tol, max_it,
                               precond=O.PREC_JACOBI if jacobi else O.PREC_NONE)
        xr, iters, conv = R.bicgstab2(rp, cols, vals, rhs, x0, tol, max_it, jacobi=jacobi)
    finally:
        O.set_threads(threads)
    assert info["iters"] == iters
    assert bool(info["converged"]) == conv
    assert np.array_equal(xo, xr), np.max(np.abs(xo - xr))
    return iters, conv


@pytest.mark.parametrize("seed", range(12))
def test_bicgstab2_matches_reference_solver(seed):
    """Seeded systems of the assembly above, from diagonally dominant (a few
    iterations) to diffusion-dominated (tens of iterations), with and without
    Jacobi, the stop at tol = 1e-10 ||b|| absolute as the workloads use it."""
    rng = np.random.default_rng(500 + seed)
    dim = 1 + seed % 3
    periodic = tuple(int(rng.integers(0, 2)) for _ in range(dim))
    n = tuple(int(rng.integers(6, 12 if dim == 3 else 40)) for _ in range(dim))
    og = O.make_grid(dim, n, [1.0] * dim, 2, periodic)
    phi = field(rng, og, "normal")
    D = float(10.0 ** rng.uniform(-3, 0))          # D dt / dx^2 from ~0.1 to ~1e3
    vel = tuple(float(rng.uniform(-1, 1)) for _ in range(dim)) if seed % 2 else None
    desc = O.AssemblyDesc(og, dt=1e-2, D=D, vel=vel, limiter=LIMS[seed % 5][1], bc=random_bc(rng, dim, periodic))
    diag, rhs, mask = O.assemble(desc, phi, phi)
    rp, cols, vals = O.export_csr(og, diag, mask)
    x0 = O.field_to_vector(og, phi)
    tol = 1e-10 * float(np.linalg.norm(rhs))
    for jacobi in (True, False):
        iters, conv = solve_both(rp, cols, vals, rhs, x0, tol, 2000, jacobi)
        assert conv and iters >= 1


def test_bicgstab2_edge_exits_match_reference_solver():
    """The iteration cap (unconverged return), an initial guess that already
    meets the tolerance (k = 0 without a preconditioner; with Jacobi the
    reference first replaces the guess by M^-1 x0, BiCGStab2.inl:258-261, and
    iterates again), and a loose tolerance met in the first iteration (the
    k > 1 rule)."""
    rng = np.random.default_rng(9)
    og = O.make_grid(3, (12, 12, 12), [1.0] * 3, 2, (0, 0, 0))
    phi = field(rng, og, "normal")
    bc = {f: (1, 0.5) for f in range(1, 7)}
    desc = O.AssemblyDesc(og, dt=1e-2, D=1.0, bc=bc)
    diag, rhs, mask = O.assemble(desc, phi, phi)
    rp, cols, vals = O.export_csr(og, diag, mask)
    x0 = O.field_to_vector(og, phi)
    tol = 1e-10 * float(np.linalg.norm(rhs))
    iters, conv = solve_both(rp, cols, vals, rhs, x0, tol, 3, True)
    assert not conv
    xs, _, _ = R.bicgstab2(rp, cols, vals, rhs, x0, tol, 2000, jacobi=False)
    iters, conv = solve_both(rp, cols, vals, rhs, xs, 1e3 * tol, 2000, False)
    assert conv and iters == 0
    iters, conv = solve_both(rp, cols, vals, rhs, xs, 1e3 * tol, 2000, True)
    assert conv and iters > 0
    iters, conv = solve_both(rp, cols, vals, rhs, x0, 0.5 * float(np.linalg.norm(rhs)), 2000, True)
    assert conv and iters >= 1


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_two_component_systems_interleave_as_the_reference(dim):
    """Two field components with their own boundary conditions (the
    counter-diffusion driver's setting, counter_diffusion1D.cpp:107-148:
    Dirichlet on one component where the other is Neumann), assembled by the
    reference's MatrixBlock<Grid, GO, SC, 2>, rows cell * 2 + c: the oracle's
    per-component assemblies interleaved into that numbering give the same
    CSR, right-hand side and initial guess bit for bit."""
    from tests.helpers import interleave_csr
    rng = np.random.default_rng(40 + dim)
    n = {1: (12,), 2: (7, 9), 3: (5, 6, 7)}[dim]
    periodic = {1: (0,), 2: (1, 0), 3: (0, 1, 0)}[dim]
    og = O.make_grid(dim, n, [1.0] * dim, 2, periodic)
    comps = [field(rng, og, "normal") for _ in range(2)]
    olds = [field(rng, og, "normal") for _ in range(2)]
    bc0, bc1 = {}, {}
    for q in range(dim):
        if periodic[q]:
            continue
        bc0[2 * q + 1], bc0[2 * q + 2] = (1, 1.0), (2, 0.0)
        bc1[2 * q + 1], bc1[2 * q + 2] = (2, 0.0), (1, 1.0)
    vel = tuple(float(v) for v in rng.uniform(-0.5, 0.5, size=dim))
    parts, rhs, x0 = [], [], []
    for c, bc in enumerate((bc0, bc1)):
        desc = O.AssemblyDesc(og, dt=1e-2, D=2e-3, vel=vel, limiter=O.LIM_MINMOD, bc=bc)
        diag, r, mask = O.assemble(desc, comps[c], olds[c])
        parts.append(O.export_csr(og, diag, mask))
        rhs.append(r)
        x0.append(O.field_to_vector(og, comps[c]))
    rp, cols, vals = interleave_csr(parts)
    orhs = np.stack(rhs, axis=-1).reshape(-1)
    ox0 = np.stack(x0, axis=-1).reshape(-1)
    rrp, rcols, rvals, rrhs, rx0 = R.assemble(dim, n, [1.0] * dim, periodic, np.concatenate(comps),
                                              np.concatenate(olds), dt=1e-2, D=2e-3, vel=vel, limiter="MINMOD",
                                              bc=bc0, ncomp=2, bc1=bc1)
    np.testing.assert_array_equal(rp, rrp)
    np.testing.assert_array_equal(cols, rcols)
    assert np.array_equal(vals, rvals), np.max(np.abs(vals - rvals))
    assert np.array_equal(orhs, rrhs), np.max(np.abs(orhs - rrhs))
    np.testing.assert_array_equal(ox0, rx0)
