"""ctypes wrapper around the CPU oracle (``libdare_oracle.so``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import this module; the product package ``dare_b200`` never does.

The oracle restates hpc-dave/dare's hot path (see ``dare_oracle.c`` for the
file:line citations) and is pinned against the reference's own known-answer
tests through the fixtures in ``tests/golden/``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdare_oracle.so")

C_, W, E, S, N, B, T = range(7)
BC_NONE, BC_DIRICHLET, BC_NEUMANN = 0, 1, 2
LIM_CDS, LIM_UPWIND, LIM_VANALBADA, LIM_MINMOD, LIM_VANLEER = range(5)
# time schemes of the Divergence operators (TimeDiscretizationSchemes.h:29-76)
(SCHEME_EULER_BACKWARD, SCHEME_EULER_FORWARD, SCHEME_CRANK_NICHOLSON, SCHEME_ADAMS_BASHFORTH,
 SCHEME_ADAMS_MOULTON) = range(5)
PREC_NONE, PREC_JACOBI = 0, 1


class Grid(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("num_ghost", C.c_int),
        ("n", C.c_int64 * 3),
        ("size", C.c_double * 3),
        ("periodic", C.c_int * 3),
    ]


class Assembly(C.Structure):
    _fields_ = [
        ("grid", Grid),
        ("dt", C.c_double),
        ("diffusion", C.c_int),
        ("D", C.c_double),
        ("face_D", C.c_void_p * 3),
        ("convection", C.c_int),
        ("limiter", C.c_int),
        ("vel", C.c_double * 3),
        ("face_vel", C.c_void_p * 3),
        ("bc_type", C.c_int * 6),
        ("bc_value", C.c_double * 6),
        ("scheme", C.c_int),
        ("no_fold", C.c_int),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("max_it", C.c_int),
        ("precond", C.c_int),
        ("iters", C.c_int),
        ("converged", C.c_int),
        ("status", C.c_int),
        ("res", C.c_double),
    ]


def build() -> None:
    """Compile the oracle with its Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        L = _lib
        pd = C.POINTER(C.c_double)
        L.dor_geometry.argtypes = [C.POINTER(Grid), pd, pd, pd]
        L.dor_num_cells.argtypes = [C.POINTER(Grid)]
        L.dor_num_cells.restype = C.c_int64
        L.dor_num_cells_ghosted.argtypes = [C.POINTER(Grid)]
        L.dor_num_cells_ghosted.restype = C.c_int64
        L.dor_ordinal_internal.argtypes = [C.POINTER(Grid), C.c_int64, C.c_int64, C.c_int64]
        L.dor_ordinal_internal.restype = C.c_int64
        L.dor_internal_to_local.argtypes = [C.POINTER(Grid), C.c_int64]
        L.dor_internal_to_local.restype = C.c_int64
        L.dor_global_internal_periodic.argtypes = [C.POINTER(Grid), C.c_int64, C.c_int64, C.c_int64]
        L.dor_global_internal_periodic.restype = C.c_int64
        L.dor_limiter.argtypes = [C.c_int, C.c_double]
        L.dor_limiter.restype = C.c_double
        L.dor_diffusion_n0d1.argtypes = [C.c_double, C.c_double, C.c_int]
        L.dor_diffusion_n0d1.restype = C.c_double
        L.dor_exchange_halo.argtypes = [C.POINTER(Grid), C.c_void_p]
        L.dor_copy_to_field.argtypes = [C.POINTER(Grid), C.c_void_p, C.c_void_p]
        L.dor_field_to_vector.argtypes = [C.POINTER(Grid), C.c_void_p, C.c_void_p]
        L.dor_assemble.argtypes = [C.POINTER(Assembly), C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
        L.dor_assemble.restype = C.c_int
        L.dor_csr_nnz.argtypes = [C.POINTER(Grid), C.c_void_p]
        L.dor_csr_nnz.restype = C.c_int64
        L.dor_export_csr.argtypes = [C.POINTER(Grid), C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        L.dor_spmv.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.dor_norm2.argtypes = [C.c_int64, C.c_void_p]
        L.dor_norm2.restype = C.c_double
        L.dor_bicgstab2.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.POINTER(SolveInfo)]
        L.dor_bicgstab2.restype = C.c_int
        L.dor_num_threads.restype = C.c_int
        L.dor_set_threads.argtypes = [C.c_int]
        L.dor_unet_num_params.restype = C.c_int64
        L.dor_unet_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.dor_unet_forward.restype = C.c_int
        L.dor_unet_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p]
        L.dor_unet_loss_grad.restype = C.c_int
    return _lib


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def make_grid(dim, n, size=None, num_ghost=2, periodic=None) -> Grid:
    g = Grid()
    g.dim = dim
    g.num_ghost = num_ghost
    nn = list(n) + [1] * (3 - len(n))
    ss = list(size if size is not None else [1.0] * dim) + [1.0] * (3 - (len(size) if size is not None else dim))
    pp = list(periodic if periodic is not None else [0] * dim) + [0] * (3 - (len(periodic) if periodic is not None else dim))
    for d in range(3):
        g.n[d] = int(nn[d]) if d < dim else 1
        g.size[d] = float(ss[d])
        g.periodic[d] = int(pp[d]) if d < dim else 0
    return g


def ghosted_shape(g: Grid):
    return tuple(int(g.n[d]) + (2 * g.num_ghost if d < g.dim else 0) for d in range(3))


def geometry(g: Grid):
    dx = (C.c_double * 3)()
    vol = C.c_double()
    area = (C.c_double * 3)()
    lib().dor_geometry(C.byref(g), dx, C.byref(vol), area)
    return list(dx), vol.value, list(area)


def exchange_halo(g: Grid, phi: np.ndarray) -> None:
    lib().dor_exchange_halo(C.byref(g), _ptr(phi))


def field_to_vector(g: Grid, phi: np.ndarray) -> np.ndarray:
    x = np.empty(int(lib().dor_num_cells(C.byref(g))), dtype=np.float64)
    lib().dor_field_to_vector(C.byref(g), _ptr(phi), _ptr(x))
    return x


def copy_to_field(g: Grid, x: np.ndarray, phi: np.ndarray) -> None:
    lib().dor_copy_to_field(C.byref(g), _ptr(np.ascontiguousarray(x, dtype=np.float64)), _ptr(phi))


def limiter(kind: int, r: float) -> float:
    return lib().dor_limiter(kind, r)


def diffusion_n0d1(tau: float, zeta: float, n_modes: int = 100) -> float:
    return lib().dor_diffusion_n0d1(tau, zeta, n_modes)


class AssemblyDesc:
    """Python-side description mirroring ``dor_assembly``; keeps arrays alive."""

    def __init__(self, grid: Grid, dt=0.0, D=None, face_D=None, vel=None, face_vel=None,
                 limiter=LIM_VANLEER, bc=None, scheme=SCHEME_EULER_BACKWARD, no_fold=False):
        self.grid = grid
        self.scheme = scheme
        self.no_fold = no_fold
        self.dt = dt
        self.D = D
        self.face_D = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                       for a in (face_D or [None, None, None])]
        self.vel = vel
        self.face_vel = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
                         for a in (face_vel or [None, None, None])]
        self.limiter = limiter
        self.bc = bc or {}

    def to_c(self) -> Assembly:
        a = Assembly()
        a.grid = self.grid
        a.dt = self.dt
        if any(x is not None for x in self.face_D):
            a.diffusion = 2
            for d in range(3):
                a.face_D[d] = None if self.face_D[d] is None else self.face_D[d].ctypes.data
        elif self.D is not None:
            a.diffusion = 1
            a.D = float(self.D)
        if any(x is not None for x in self.face_vel):
            a.convection = 2
            for d in range(3):
                a.face_vel[d] = None if self.face_vel[d] is None else self.face_vel[d].ctypes.data
        elif self.vel is not None:
            a.convection = 1
            for d in range(len(self.vel)):
                a.vel[d] = float(self.vel[d])
        a.limiter = self.limiter
        a.scheme = self.scheme
        a.no_fold = int(self.no_fold)
        for face, (kind, value) in self.bc.items():
            a.bc_type[face - 1] = kind
            a.bc_value[face - 1] = value
        return a


def assemble(desc: AssemblyDesc, phi_conv: np.ndarray, phi_old: np.ndarray | None = None):
    """Returns (diag[7, ncell], rhs[ncell], mask[ncell])."""
    g = desc.grid
    n = int(lib().dor_num_cells(C.byref(g)))
    diag = np.zeros((7, n), dtype=np.float64)
    rhs = np.zeros(n, dtype=np.float64)
    mask = np.zeros(n, dtype=np.uint8)
    a = desc.to_c()
    phi_conv = np.ascontiguousarray(phi_conv, dtype=np.float64)
    phi_old = phi_conv if phi_old is None else np.ascontiguousarray(phi_old, dtype=np.float64)
    rc = lib().dor_assemble(C.byref(a), _ptr(phi_conv), _ptr(phi_old), _ptr(diag), _ptr(rhs), _ptr(mask))
    if rc != 0:
        raise ValueError("oracle: invalid assembly description")
    return diag, rhs, mask


def export_csr(g: Grid, diag: np.ndarray, mask: np.ndarray):
    n = int(lib().dor_num_cells(C.byref(g)))
    nnz = int(lib().dor_csr_nnz(C.byref(g), _ptr(mask)))
    rowptr = np.zeros(n + 1, dtype=np.int64)
    cols = np.zeros(nnz, dtype=np.int64)
    vals = np.zeros(nnz, dtype=np.float64)
    lib().dor_export_csr(C.byref(g), _ptr(np.ascontiguousarray(diag)), _ptr(mask), _ptr(rowptr),
                         _ptr(cols), _ptr(vals))
    return rowptr, cols, vals


def spmv(rowptr, cols, vals, x):
    y = np.empty(len(rowptr) - 1, dtype=np.float64)
    lib().dor_spmv(len(rowptr) - 1, _ptr(rowptr), _ptr(cols), _ptr(vals),
                   _ptr(np.ascontiguousarray(x, dtype=np.float64)), _ptr(y))
    return y


def bicgstab2(rowptr, cols, vals, b, x0, tol, max_it=5000, precond=PREC_JACOBI):
    """Runs the restated BiCGStab2 (absolute-norm stop). Returns (x, info dict)."""
    x = np.ascontiguousarray(x0, dtype=np.float64).copy()
    info = SolveInfo()
    info.tol = tol
    info.max_it = max_it
    info.precond = precond
    rc = lib().dor_bicgstab2(len(rowptr) - 1, _ptr(rowptr), _ptr(cols), _ptr(vals),
                             _ptr(np.ascontiguousarray(b, dtype=np.float64)), _ptr(x), C.byref(info))
    if rc != 0:
        raise MemoryError("oracle bicgstab2 failed to allocate")
    return x, dict(iters=info.iters, converged=bool(info.converged), status=info.status, res=info.res)


def num_threads() -> int:
    return lib().dor_num_threads()


def set_threads(n: int) -> None:
    lib().dor_set_threads(n)


# ---- learned linear preconditioner (dare_oracle_unet.c) ----------------------
UNET_LAYERS = (("enc0", 0, 1, 16), ("enc1", 1, 16, 32), ("enc2", 2, 32, 64), ("enc3", 3, 64, 64),
               ("dec3", 3, 64, 64), ("dec2", 2, 64, 32), ("dec1", 1, 32, 16), ("dec0", 0, 16, 1))
UNET_ACTS = (("S0", 0, 16), ("P1", 1, 16), ("S1", 1, 32), ("P2", 2, 32), ("S2", 2, 64), ("P3", 3, 64),
             ("E3", 3, 64))


def unet_num_params() -> int:
    return int(lib().dor_unet_num_params())


def unet_layer_slices():
    """name -> (slice into the flat parameter vector, (27, cout, cin))."""
    out, off = {}, 0
    for name, _, cin, cout in UNET_LAYERS:
        m = 27 * cin * cout
        out[name] = (slice(off, off + m), (27, cout, cin))
        off += m
    return out


def unet_forward(n, w, u, bf16=True, with_acts=False):
    """z = u + U(u) (float64); optionally the activations S0..E3 as a dict."""
    n3 = np.ascontiguousarray(n, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    u = np.ascontiguousarray(u, dtype=np.float64).ravel()
    z = np.empty_like(u)
    acts = None
    if with_acts:
        cells = [int(np.prod([x >> l for x in n])) for l in range(4)]
        acts = np.empty(sum(cells[l] * c for _, l, c in UNET_ACTS), dtype=np.float64)
    rc = lib().dor_unet_forward(_ptr(n3), _ptr(w), _ptr(u), int(bf16), _ptr(z), _ptr(acts))
    if rc:
        raise ValueError("oracle unet: bad grid")
    if not with_acts:
        return z
    res, off = {}, 0
    for name, l, c in UNET_ACTS:
        m = cells[l] * c
        res[name] = acts[off:off + m].reshape(cells[l], c)
        off += m
    return z, res


def unet_loss_grad(n, w, r, e, bf16=True, want_grad=True):
    """Mean relative squared error over the pairs (rows of r, e) and its gradient."""
    n3 = np.ascontiguousarray(n, dtype=np.int32)
    w = np.ascontiguousarray(w, dtype=np.float32)
    r = np.ascontiguousarray(r, dtype=np.float64)
    e = np.ascontiguousarray(e, dtype=np.float64)
    count = r.shape[0] if r.ndim == 2 else 1
    loss = C.c_double(0.0)
    grad = np.empty(unet_num_params(), dtype=np.float64) if want_grad else None
    rc = lib().dor_unet_loss_grad(_ptr(n3), _ptr(w), _ptr(r), _ptr(e), count, int(bf16), C.byref(loss), _ptr(grad))
    if rc:
        raise ValueError("oracle unet: bad grid")
    return loss.value, grad
