"""Shared test helpers: oracle-side time loop and the reference's solver
functors (test infrastructure; used by tests only)."""
import numpy as np

from oracle import oracle as O


def oracle_grid(case, ng=2):
    n = case["n"]
    dim = len([x for x in n])
    return O.make_grid(dim, n, case.get("size"), ng, case.get("periodic"))


def oracle_assembly(og, case, face_D=None):
    bc = {int(k): v for k, v in case.get("bc", {}).items()}
    lim = {"CDS": O.LIM_CDS, "UPWIND": O.LIM_UPWIND, "VANALBADA": O.LIM_VANALBADA, "MINMOD": O.LIM_MINMOD,
           "VANLEER": O.LIM_VANLEER}[case.get("limiter", "VANLEER")]
    fv = case.get("face_vel")
    fv = None if fv is None else [np.ascontiguousarray(np.asarray(a), dtype=np.float64) for a in fv]
    scheme = {"EULER_BACKWARD": O.SCHEME_EULER_BACKWARD, "EULER_FORWARD": O.SCHEME_EULER_FORWARD,
              "CRANK_NICHOLSON": O.SCHEME_CRANK_NICHOLSON, "ADAMS_BASHFORTH": O.SCHEME_ADAMS_BASHFORTH,
              "ADAMS_MOULTON": O.SCHEME_ADAMS_MOULTON}[case.get("scheme", "EULER_BACKWARD")]
    return O.AssemblyDesc(og, dt=case.get("dt", 0.0), D=case.get("D"), face_D=face_D, vel=case.get("vel"),
                          face_vel=fv, limiter=lim, bc=bc, scheme=scheme)


def oracle_timeloop(case, steps, precond=O.PREC_JACOBI, face_D=None, max_it=5000):
    """The reference's driver loop on the CPU oracle: Build, Solve, CopyTo,
    ExchangeHaloCells, CopyDataVectorsToOldTimeStep (counter_diffusion1D.cpp:170-217)."""
    og = oracle_grid(case)
    desc = oracle_assembly(og, case, face_D)
    phi = np.ascontiguousarray(np.asarray(case["phi0"], dtype=np.float64).reshape(-1)).copy()
    old = phi.copy()
    history, iters = [], []
    for _ in range(steps):
        diag, rhs, mask = O.assemble(desc, phi, old)
        rowptr, cols, vals = O.export_csr(og, diag, mask)
        x0 = O.field_to_vector(og, phi)
        tol = case.get("rel_tol", 1e-10) * float(np.linalg.norm(rhs))
        x, info = O.bicgstab2(rowptr, cols, vals, rhs, x0, tol=tol, max_it=max_it, precond=precond)
        O.copy_to_field(og, x, phi)
        O.exchange_halo(og, phi)
        old[:] = phi
        history.append(phi.copy())
        iters.append(info["iters"])
    return history, iters


def ref_timeloop(case, steps, max_it=5000):
    """The same driver loop with the reference's own assembly and BiCGStab2
    (oracle/_ref: its Grid/Cartesian, Equations, MatrixBlock and BiCGStab2
    code) for a case without face fields (scalar D, constant or no velocity).
    The copy back and the periodic ghost fill are the oracle's.  Returns the
    field history, the iterations and the seconds spent in assembly and
    solve."""
    import time

    from oracle import ref as R
    og = oracle_grid(case)
    n = tuple(case["n"])
    dim = len(n)
    lim = case.get("limiter", "VANLEER")
    phi = np.ascontiguousarray(np.asarray(case["phi0"], dtype=np.float64).reshape(-1)).copy()
    old = phi.copy()
    bc = {int(k): v for k, v in case.get("bc", {}).items()}
    history, iters, secs = [], [], 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        rp, cols, vals, rhs, x0 = R.assemble(dim, n, case.get("size", (1.0,) * dim), case.get("periodic", (0,) * dim),
                                             phi, old, dt=case.get("dt", 0.0), D=case.get("D"), vel=case.get("vel"),
                                             limiter=lim, bc=bc)
        tol = case.get("rel_tol", 1e-10) * float(np.linalg.norm(rhs))
        x, it, conv = R.bicgstab2(rp, cols, vals, rhs, x0, tol, max_it, jacobi=True)
        secs += time.perf_counter() - t0
        O.copy_to_field(og, x, phi)
        O.exchange_halo(og, phi)
        old[:] = phi
        history.append(phi.copy())
        iters.append(it)
    return history, iters, secs


def interior(phi, shape, ng=2, dim=3):
    a = np.asarray(phi).reshape(shape)
    sl = tuple(slice(ng, s - ng) if d < dim else slice(None) for d, s in enumerate(shape))
    return a[sl]


def rel_l2(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


COEF_RTOL = 1e-13   # assembled FP64 coefficients, relative


def assert_coef_close(got, ref, rtol=COEF_RTOL):
    """Assembled coefficients within `rtol` relative: per entry
    |got - ref| <= rtol |ref| + rtol max|ref of that slot| (the second term
    covers entries that are sums with cancellation, e.g. a deferred-correction
    rhs where phi_old = 0).  NaN where the reference has NaN (VANALBADA at
    r = +-inf)."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape
    rows = ref.reshape(-1, ref.shape[-1]) if ref.ndim > 1 else ref[None, :]
    grows = got.reshape(rows.shape)
    for g, r in zip(grows, rows):
        fin = np.isfinite(r)
        scale = np.abs(r[fin]).max() if fin.any() else 0.0
        np.testing.assert_allclose(g, r, rtol=rtol, atol=rtol * scale, equal_nan=True)


def profile_functor_diag(dim, n, west=0.0, east=1.0):
    """SoA coefficients of test_integration_Cartesian_Trilinos.cpp SolveScalar(X)
    (1D :99-130, 2D :245-294, 3D :602-672): centre 2*dim, neighbours -1,
    Dirichlet mirror on W/E, Neumann on the other faces; removed slots 0."""
    nn = list(n) + [1] * (3 - dim)
    N = nn[0] * nn[1] * nn[2]
    diag = np.zeros((7, N))
    rhs = np.zeros(N)
    x0 = np.zeros(N)
    idx = np.indices(nn).reshape(3, -1)
    diag[0] = 2.0 * dim
    for d in range(dim):
        lo, hi = 2 * d + 1, 2 * d + 2
        at_lo = idx[d] == 0
        at_hi = idx[d] == nn[d] - 1
        diag[lo] = np.where(at_lo, 0.0, -1.0)
        diag[hi] = np.where(at_hi, 0.0, -1.0)
        if d == 0:
            diag[0] += at_lo * 1.0 + at_hi * 1.0
            rhs = np.where(at_lo, 2.0 * west, rhs)
            rhs = np.where(at_hi, 2.0 * east, rhs)
            x0 = np.where(at_lo, west, x0)
            x0 = np.where(at_hi, east, x0)
        else:
            diag[0] -= at_lo * 1.0 + at_hi * 1.0
    return diag, rhs, x0


def coupled_components_diag(ncell=23, ncomp=4):
    """MatrixSystem/test/test_TrilinosSolver.cpp:120-165 as a 2D structured
    grid (cells along x, interleaved components along y)."""
    N = ncell * ncomp
    diag = np.zeros((7, N))
    rhs = np.zeros(N)
    x0 = np.full(N, 0.5)
    node = np.repeat(np.arange(ncell), ncomp)
    comp = np.tile(np.arange(ncomp), ncell)
    left, right = node == 0, node == ncell - 1
    diag[0] = np.where(left | right, 3.0, 2.0)
    diag[1] = np.where(left, 0.0, -1.0)   # WEST  (row - N)
    diag[2] = np.where(right, 0.0, -1.0)  # EAST  (row + N)
    rhs = np.where(right, 2.0, 0.0)
    x0 = np.where(left, 0.0, np.where(right, 1.0, x0))
    diag[3] = np.where(comp == 0, 0.0, -1.0)           # SOUTH (row - 1)
    diag[4] = np.where(comp == ncomp - 1, 0.0, -1.0)   # NORTH (row + 1)
    diag[0] += (comp != 0) * 1.0 + (comp != ncomp - 1) * 1.0
    return diag, rhs, x0


def diag_to_csr(dim, n, diag, periodic=None):
    """CSR of SoA coefficients with the Finalize pattern (removed = out of range)."""
    og = O.make_grid(dim, n, None, 2, periodic)
    nn = list(n) + [1] * (3 - dim)
    idx = np.indices(nn).reshape(3, -1)
    mask = np.ones(idx.shape[1], dtype=np.uint8)
    pp = list(periodic or [0] * dim) + [0] * (3 - dim)
    for d in range(dim):
        lo = np.ones(idx.shape[1], dtype=bool) if pp[d] else idx[d] > 0
        hi = np.ones(idx.shape[1], dtype=bool) if pp[d] else idx[d] < nn[d] - 1
        mask |= (lo.astype(np.uint8) << (2 * d + 1)) | (hi.astype(np.uint8) << (2 * d + 2))
    return O.export_csr(og, np.ascontiguousarray(diag), mask)


def interleave_csr(csrs):
    """Rows cell * N + c and columns neighbour * N + c from one CSR per component
    (MatrixBlock_Cartesian.inl:127-240: no coupling between components)."""
    N = len(csrs)
    rp0 = csrs[0][0]
    ncell = rp0.size - 1
    rows, cols, vals = [], [], []
    for cell in range(ncell):
        for c, (rp, co, va) in enumerate(csrs):
            a, b = rp[cell], rp[cell + 1]
            rows.append(b - a)
            cols.append(co[a:b] * N + c)
            vals.append(va[a:b])
    rowptr = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    return rowptr, np.concatenate(cols).astype(np.int64), np.concatenate(vals)


# ---- composed functors (dare_assemble_terms) on the oracle -----------------------
ORACLE_LIM = {"CDS": O.LIM_CDS, "UPWIND": O.LIM_UPWIND, "VANALBADA": O.LIM_VANALBADA, "MINMOD": O.LIM_MINMOD,
              "VANLEER": O.LIM_VANLEER}


def fold_faces(og_n, periodic, dim, diag, rhs, bc):
    """The boundary folding of counter_diffusion1D.cpp:123-146 on one
    component's coefficients, faces in the order W, E, S, N, B, T: Dirichlet
    C -= X, rhs -= 2 bc X; Neumann C += X; the face's coefficient removed."""
    n = list(og_n) + [1] * (3 - len(og_n))
    idx = np.indices(n).reshape(3, -1)
    for d in range(dim):
        if periodic[d]:
            continue
        for side in (0, 1):
            face = 2 * d + 1 + side
            on = idx[d] == 0 if side == 0 else idx[d] == n[d] - 1
            X = diag[face][on].copy()
            kind, value = bc[face]
            if kind == O.BC_DIRICHLET:
                diag[0][on] -= X
                rhs[on] -= 2. * value * X
            else:
                diag[0][on] += X
            diag[face][on] = 0.0
    return diag, rhs


def oracle_terms(og, case, terms, phis, olds, bcs):
    """A composed functor on the oracle, per component: each term's unfolded
    contribution (the oracle's parts enter as DDT +, convection +, diffusion -,
    i.e. mb -= div(D grad)) combined in order -- SET starts afresh, ADD adds,
    SUB adds the negative (MatrixBlock_Cartesian.inl:480-593) -- then the
    component's boundary folding.  Returns diag (7, ncell * N) and rhs with
    rows cell * N + c, as the system exports them, the per-component
    coefficients and the pattern mask."""
    N = len(phis)
    dim = len(case["n"])
    per = list(case.get("periodic") or [0] * dim) + [0] * (3 - dim)
    neutral = {f: (O.BC_NEUMANN, 0.0) for f in range(1, 7)}
    diags, rhss = [], []
    for c in range(N):
        acc_d = acc_r = None
        for t in terms:
            if t["component"] not in (-1, c):
                continue
            kind = t["kind"]
            if kind == "COEFFS":   # the caller's own values: 7 slot arrays (None: 0) and the rhs
                ncell = int(np.prod(case["n"]))
                d = np.stack([np.zeros(ncell) if a is None else np.asarray(a, dtype=np.float64)
                              for a in t["coef"]])
                r = np.zeros(ncell) if t.get("rhs") is None else np.asarray(t["rhs"], dtype=np.float64).copy()
                native = 1.0
            else:
                desc = O.AssemblyDesc(og, dt=t.get("dt", 0.0) if kind == "DDT" else 0.0,
                                      D=t.get("D", 1.0) if kind == "DIFFUSION" else None,
                                      vel=t.get("vel") if kind == "CONVECTION" else None,
                                      limiter=ORACLE_LIM[t.get("limiter", "VANLEER")], bc=neutral, no_fold=True)
                d, r, mask = O.assemble(desc, np.ascontiguousarray(phis[c]), np.ascontiguousarray(olds[c]))
                native = -1.0 if kind == "DIFFUSION" else 1.0
            want = -1.0 if t["op"] == "SUB" else 1.0
            if want != native:
                d, r = -d, -r
            if acc_d is None or t["op"] == "SET":
                acc_d, acc_r = d.copy(), r.copy()
            else:
                acc_d += d
                acc_r += r
        ncell = int(np.prod(case["n"]))
        if acc_d is None:
            acc_d, acc_r = np.zeros((7, ncell)), np.zeros(ncell)
        acc_d, acc_r = fold_faces(case["n"], per, dim, acc_d, acc_r, bcs[c])
        diags.append(acc_d)
        rhss.append(acc_r)
    ncell = diags[0].shape[1]
    diag = np.stack(diags, axis=-1).reshape(7, ncell * N)
    rhs = np.stack(rhss, axis=-1).reshape(-1)
    ghost = np.zeros(int(np.prod(O.ghosted_shape(og))))
    mask = O.assemble(O.AssemblyDesc(og, dt=1.0, bc=neutral), ghost)[2]   # the pattern: removed boundary faces
    return diag, rhs, (diags, rhss), mask
