"""Staggered grids (dare_grid_create_staggered), the reference's staggered
representation (CartesianRepresentation.inl:33-76): one more cell along a
staggered, non-periodic direction, the base grid's cell width, the domain
shifted by half a cell.  The reference's staggered solves are reproduced --
test_integration_Cartesian_Trilinos.cpp SolveStaggered (1-D, :155-222),
SolveStaggeredX / SolveStaggeredY (2-D, :410-582) and SolveStaggeredZ (3-D,
:697-) -- with their functors (identity rows on the two ends of the profile
direction, a Laplacian with the missing neighbours dropped elsewhere), three
components, BiCGStab2 to 1e-14: the linear profile within 1e-8 and the
oracle's solve of the exported matrix within 1e-9."""
import numpy as np
import pytest

import dare_b200 as D
from oracle import oracle as O
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

N_COMP = 3   # IntegrationCartesianTrilinos::N


@pytest.fixture(scope="module")
def ctx():
    return D.Context(0)


def staggered_functor(nn, dim, prof, lo, hi):
    """The functor of the reference's staggered solves on the representation
    of size nn: cells on the two ends of direction `prof` are identity rows
    (rhs and initial guess the end value); every other cell has centre 2 dim
    minus one per missing neighbour, -1 for each present neighbour, rhs 0."""
    n3 = list(nn) + [1] * (3 - dim)
    ncell = int(np.prod(n3))
    idx = np.indices(n3).reshape(3, -1)
    diag = np.zeros((7, ncell))
    rhs = np.zeros(ncell)
    x0 = np.zeros(ncell)
    lo_edge = idx[prof] == 0
    hi_edge = idx[prof] == n3[prof] - 1
    inner = ~(lo_edge | hi_edge)
    diag[0] = np.where(inner, 2.0 * dim, 1.0)
    for d in range(dim):
        at_lo, at_hi = idx[d] == 0, idx[d] == n3[d] - 1
        if d != prof:
            diag[0] -= inner * (at_lo * 1.0 + at_hi * 1.0)
        diag[2 * d + 1] = np.where(inner & ~at_lo, -1.0, 0.0)
        diag[2 * d + 2] = np.where(inner & ~at_hi, -1.0, 0.0)
    rhs = np.where(lo_edge, lo, np.where(hi_edge, hi, 0.0))
    x0 = rhs.copy()
    return diag, rhs, x0, idx


CASES = [
    # (name, base resolution, size, staggered, profile direction)
    ("SolveStaggered", (20,), (1.0,), (1,), 0),
    ("SolveStaggeredX", (20, 21), (1.0, 2.0), (1, 0), 0),
    ("SolveStaggeredY", (20, 21), (1.0, 2.0), (0, 1), 1),
    ("SolveStaggeredZ", (20, 21, 22), (1.0, 2.0, 3.0), (1, 0, 0), 2),   # opt(1, 0) as in the reference
]


@pytest.mark.parametrize("name,n,size,stag,prof", CASES)
@pytest.mark.parametrize("precond", ["NONE", "JACOBI"])
def test_reference_staggered_solves(ctx, name, n, size, stag, prof, precond):
    dim = len(n)
    g = D.Grid(ctx, n, size, 2, None, staggered=stag)
    nn = [n[d] + stag[d] for d in range(dim)]
    assert list(g.n[:dim]) == nn
    for d in range(dim):
        assert g.dx[d] == pytest.approx(size[d] / n[d], rel=0, abs=0)
        assert g.origin[d] == (-0.5 * g.dx[d] if stag[d] else 0.0)
    diag, rhs, x0, idx = staggered_functor(nn, dim, prof, 0.0, 1.0)
    ncell = diag.shape[1]
    inter = lambda a: np.repeat(a[..., None], N_COMP, axis=-1).reshape(*a.shape[:-1], ncell * N_COMP)
    s = D.MatrixSystem(g, components=N_COMP)
    s.set_coefficients(inter(diag), inter(rhs), inter(x0))
    rep = D.BiCGStab2({"Convergence Tolerance": 1e-14, "Maximum Iterations": 5000}, precond=precond).solve(s)
    assert rep["converged"], rep
    x = s.solution().reshape(ncell, N_COMP)
    d_phi = 1.0 / (nn[prof] - 1)
    for c in range(N_COMP):
        assert np.max(np.abs(x[:, c] - idx[prof] * d_phi)) < 1e-8, (name, c)
    rp, cols, vals = s.export_csr()
    ox, info = O.bicgstab2(rp, cols, vals, inter(rhs), inter(x0), 1e-14, 5000,
                           O.PREC_JACOBI if precond == "JACOBI" else O.PREC_NONE)
    assert info["converged"]
    assert rel_l2(x.reshape(-1), ox) < 1e-9


def test_periodic_direction_is_not_staggered(ctx):
    """A periodic direction gains no cell and keeps its origin
    (CartesianRepresentation.inl:67-76 skips periodic directions)."""
    g = D.Grid(ctx, (12, 10), (1.0, 1.0), 2, (1, 0), staggered=(1, 1))
    assert g.n[:2] == (12, 11)
    assert g.origin[0] == 0.0 and g.origin[1] == -0.05


def test_staggered_vtk_node_coordinates(ctx, tmp_path):
    """The VTK writer places the nodes of a staggered grid half a cell lower
    (offset_size - num_ghost dx, VTKOptions_Cartesian.h:160-162)."""
    import xml.etree.ElementTree as ET
    from tests.test_vtk_writer import _decode
    n, size = (8, 6), (1.0, 1.5)
    g = D.Grid(ctx, n, size, 2, None, staggered=(1, 0))
    f = D.Field(g, 1)
    f.upload(np.zeros(g.num_cells_ghosted), 0)
    D.write_vtk([f], ["phi"], str(tmp_path), "Grid_X", 0)
    root = ET.parse(str(tmp_path / "Grid_X_0" / "Grid_X_0_0.vts")).getroot()
    pts = _decode(root.find("StructuredGrid").find("Piece").find("Points").find("DataArray").text,
                  np.float32).reshape(-1, 3)
    dx, dy = size[0] / n[0], size[1] / n[1]
    assert pts[0, 0] == np.float32(-0.5 * dx - 2 * dx)   # staggered direction: half a cell lower
    assert pts[0, 1] == np.float32(-2 * dy)               # the other: as on the base grid
    assert pts[1, 0] == np.float32(-0.5 * dx - dx)
