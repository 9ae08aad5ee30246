"""The oracle's assembly against the reference's own code.

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
Neumann faces.  The library is built where the reference's sources are
present (``make -C oracle ref``).
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
