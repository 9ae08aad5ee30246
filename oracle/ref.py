"""ctypes binding of oracle/_ref/libdare_ref.so: the reference's own assembly
code (its Grid/Cartesian, Equations, Data and MatrixSystem headers) and its
BiCGStab2 solver, compiled against the single-rank stand-ins in
oracle/ref_shim/, used to check the C restatement in dare_oracle.c.  Test
infrastructure only; built by ``make -C oracle ref`` where the reference's
sources are present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libdare_ref.so")

LIMITERS = {"CDS": 0, "UPWIND": 1, "VANALBADA": 2, "MINMOD": 3, "VANLEER": 4}
SCHEMES = {"EULER_BACKWARD": 0, "EULER_FORWARD": 1, "CRANK_NICHOLSON": 2, "ADAMS_BASHFORT": 3}


class Desc(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int64 * 3), ("L", C.c_double * 3), ("periodic", C.c_int * 3),
                ("dt", C.c_double), ("diffusion", C.c_int), ("D", C.c_double),
                ("face_D", C.c_void_p * 3), ("convection", C.c_int), ("vel", C.c_double * 3),
                ("limiter", C.c_int), ("scheme", C.c_int), ("bc_type", C.c_int * 6), ("bc_value", C.c_double * 6),
                ("ncomp", C.c_int), ("bc_type1", C.c_int * 6), ("bc_value1", C.c_double * 6)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(LIB_PATH)
        _lib.dref_assemble.restype = C.c_int
        _lib.dref_assemble.argtypes = [C.POINTER(Desc)] + [C.c_void_p] * 7 + [C.c_int64]
        _lib.dref_bicgstab2.restype = C.c_int
        _lib.dref_bicgstab2.argtypes = [C.c_int64] + [C.c_void_p] * 5 + [C.c_double, C.c_int, C.c_int,
                                                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return _lib


def assemble(dim, n, L, periodic, phi_conv, phi_old, dt=0.0, D=None, face_D=None, vel=None,
             limiter="VANLEER", scheme="EULER_BACKWARD", bc=None, ncomp=1, bc1=None):
    """CSR (rowptr, cols, vals), rhs and initial guess of one implicit step,
    assembled by the reference's code.  bc: {face 1..6: (1 Dirichlet | 2
    Neumann, value)}, bc1 the same for component 1 when ncomp = 2; fields
    are ghosted (two layers) in the oracle's layout, component after
    component; rows are cell * ncomp + component."""
    d = Desc()
    d.dim = dim
    for q in range(3):
        d.n[q] = int(n[q]) if q < dim else 1
        d.L[q] = float(L[q]) if q < dim else 1.0
        d.periodic[q] = int(periodic[q]) if q < dim else 0
    d.dt = dt
    keep = []
    if face_D is not None:
        d.diffusion = 2
        for q in range(dim):
            a = np.ascontiguousarray(face_D[q], dtype=np.float64)
            keep.append(a)
            d.face_D[q] = a.ctypes.data
    elif D is not None:
        d.diffusion = 1
        d.D = float(D)
    if vel is not None:
        d.convection = 1
        for q in range(dim):
            d.vel[q] = float(vel[q])
    d.limiter = LIMITERS[limiter]
    d.scheme = SCHEMES[scheme]
    for face, (kind, value) in (bc or {}).items():
        d.bc_type[face - 1] = kind
        d.bc_value[face - 1] = value
    d.ncomp = ncomp
    for face, (kind, value) in (bc1 or {}).items():
        d.bc_type1[face - 1] = kind
        d.bc_value1[face - 1] = value
    ncell = int(np.prod([d.n[q] for q in range(3)])) * ncomp
    phi_conv = np.ascontiguousarray(phi_conv, dtype=np.float64)
    phi_old = np.ascontiguousarray(phi_old, dtype=np.float64)
    rowptr = np.zeros(ncell + 1, dtype=np.int64)
    cap = 7 * ncell
    cols = np.zeros(cap, dtype=np.int64)
    vals = np.zeros(cap, dtype=np.float64)
    rhs = np.zeros(ncell, dtype=np.float64)
    x0 = np.zeros(ncell, dtype=np.float64)
    rc = lib().dref_assemble(C.byref(d), phi_conv.ctypes.data, phi_old.ctypes.data, rowptr.ctypes.data,
                             cols.ctypes.data, vals.ctypes.data, rhs.ctypes.data, x0.ctypes.data, cap)
    if rc != 0:
        raise ValueError(f"reference assembly failed ({rc})")
    nnz = int(rowptr[-1])
    return rowptr, cols[:nnz], vals[:nnz], rhs, x0


def bicgstab2(rowptr, cols, vals, b, x0, tol, max_it=5000, jacobi=True):
    """The reference's BiCGStab2::solve on a CSR system: (x, iterations,
    converged).  tol is absolute (its RNORM criterion)."""
    n = len(rowptr) - 1
    rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True)
    iters, conv = C.c_int(0), C.c_int(0)
    rc = lib().dref_bicgstab2(n, rowptr.ctypes.data, cols.ctypes.data, vals.ctypes.data, b.ctypes.data,
                              x.ctypes.data, float(tol), int(max_it), int(bool(jacobi)), C.byref(iters),
                              C.byref(conv))
    if rc != 0:
        raise RuntimeError("the reference's BiCGStab2 threw")
    return x, iters.value, bool(conv.value)
