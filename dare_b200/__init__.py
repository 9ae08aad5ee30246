"""dare_b200 -- B200-native finite-volume hot path of hpc-dave/dare.

Python binding of the C ABI in ``include/dare_gpu.h`` (``libdare_gpu.so``,
hand-written CUDA for sm_100a).  There is no CPU fallback: every object here
drives device kernels, and importing a handle class without the built library
raises ``RuntimeError``.

The classes mirror the reference's host API for the path:

=====================  ====================================================
reference (C++)         here
=====================  ====================================================
Grid::Cartesian<Dim>    :class:`Grid`
Data::Field             :class:`Field` (time levels of ghosted GridVectors)
Matrix::Trilinos<SC>    :class:`MatrixSystem` (``build``, ``copy_to``, CSR export)
Matrix::BiCGStab2       :class:`BiCGStab2` (``"Convergence Tolerance"``,
                        ``"Maximum Iterations"`` parameter names)
=====================  ====================================================
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdare_gpu.so")

CENTER, WEST, EAST, SOUTH, NORTH, BOTTOM, TOP = range(7)
BC_PERIODIC, BC_DIRICHLET, BC_NEUMANN = 0, 1, 2
LIMITER = {"CDS": 0, "UPWIND": 1, "VANALBADA": 2, "MINMOD": 3, "VANLEER": 4}
# time schemes of the div(...) terms (Equations/TimeDiscretizationSchemes.h)
SCHEME = {"EULER_BACKWARD": 0, "EULER_FORWARD": 1, "CRANK_NICHOLSON": 2, "ADAMS_BASHFORTH": 3,
          "ADAMS_MOULTON": 4}
PREC_NONE, PREC_JACOBI = 0, 1
PRECISION_FP64, PRECISION_FP32_REFINE = 0, 1
SOLVE_STATUS = {0: "converged", 1: "max_iterations", 2: "breakdown", 3: "nan"}
KERNEL_IDS = {"assemble": 0, "step1": 3, "step2": 4, "step3": 5, "step4": 6, "step5": 7,
              # the FP32 inner iterations of the refinement solve
              "fp32_step1": 9, "fp32_step2": 10, "fp32_step3": 11, "fp32_step4": 12, "fp32_step5": 13}


class GridInfo(C.Structure):
    _fields_ = [("dim", C.c_int), ("num_ghost", C.c_int), ("n", C.c_int64 * 3), ("n_ghosted", C.c_int64 * 3),
                ("num_cells", C.c_int64), ("num_cells_ghosted", C.c_int64), ("dx", C.c_double * 3),
                ("volume", C.c_double), ("area", C.c_double * 3), ("periodic", C.c_int * 3),
                ("staggered", C.c_int * 3), ("origin", C.c_double * 3)]


class AssemblyDesc(C.Structure):
    _fields_ = [("dt", C.c_double), ("diffusion", C.c_int), ("D", C.c_double), ("face_D", C.c_void_p * 3),
                ("convection", C.c_int), ("limiter", C.c_int), ("vel", C.c_double * 3),
                ("face_vel", C.c_void_p * 3), ("scheme", C.c_int)]


class TermDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("op", C.c_int), ("component", C.c_int), ("dt", C.c_double), ("D", C.c_double),
                ("face_D", C.c_void_p * 3), ("vel", C.c_double * 3), ("face_vel", C.c_void_p * 3),
                ("limiter", C.c_int), ("scheme", C.c_int), ("coef", C.c_void_p * 7), ("coef_rhs", C.c_void_p)]


class SolverParams(C.Structure):
    _fields_ = [("tol", C.c_double), ("max_it", C.c_int), ("precond", C.c_int), ("precision", C.c_int),
                ("inner_rel_tol", C.c_double), ("inner_max_it", C.c_int), ("max_refinements", C.c_int),
                ("check_every", C.c_int), ("compute_true_residual", C.c_int), ("tol_relative", C.c_int)]


class SolveReport(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("status", C.c_int), ("breakdown_step", C.c_int),
                ("res_abs", C.c_double), ("true_res_abs", C.c_double), ("b_norm", C.c_double),
                ("refinements", C.c_int), ("inner_iters", C.c_int), ("fallback_used", C.c_int),
                ("tol_abs", C.c_double)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["status_name"] = SOLVE_STATUS.get(self.status, str(self.status))
        return d


# every symbol declared in include/dare_gpu.h: (name, restype, argtypes)
_P = C.c_void_p
_SIGS = [
    ("dare_ctx_create", C.c_int, [C.c_int, C.POINTER(_P)]),
    ("dare_ctx_destroy", C.c_int, [_P]),
    ("dare_ctx_set_stream", C.c_int, [_P, _P]),
    ("dare_ctx_get_stream", _P, [_P]),
    ("dare_ctx_synchronize", C.c_int, [_P]),
    ("dare_ctx_last_error", C.c_char_p, [_P]),
    ("dare_ctx_launch_count", C.c_int64, [_P]),
    ("dare_ctx_set_profiling", C.c_int, [_P, C.c_int]),
    ("dare_ctx_reset_kernel_stats", C.c_int, [_P]),
    ("dare_ctx_kernel_stats", C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("dare_ctx_timer_start", C.c_int, [_P]),
    ("dare_ctx_timer_stop", C.c_int, [_P, C.POINTER(C.c_double)]),
    ("dare_grid_create", C.c_int, [_P, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int,
                                   C.POINTER(C.c_int), C.POINTER(_P)]),
    ("dare_grid_create_staggered", C.c_int, [_P, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int,
                                             C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(_P)]),
    ("dare_grid_destroy", C.c_int, [_P]),
    ("dare_grid_get_info", C.c_int, [_P, C.POINTER(GridInfo)]),
    ("dare_field_create", C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    ("dare_field_create_n", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P)]),
    ("dare_field_num_components", C.c_int, [_P]),
    ("dare_system_create_n", C.c_int, [_P, C.c_int, C.POINTER(_P)]),
    ("dare_system_num_components", C.c_int, [_P]),
    ("dare_field_destroy", C.c_int, [_P]),
    ("dare_field_upload", C.c_int, [_P, C.c_int, _P]),
    ("dare_field_download", C.c_int, [_P, C.c_int, _P]),
    ("dare_field_device_ptr", _P, [_P, C.c_int]),
    ("dare_field_exchange_halo", C.c_int, [_P]),
    ("dare_field_copy_to_old", C.c_int, [_P]),
    ("dare_vtk_write", C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(C.c_char_p), C.c_int, C.c_char_p, C.c_char_p,
                                 C.c_int, C.c_double]),
    ("dare_vtk_write_host", C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_double), C.c_int,
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_char_p), C.c_int, C.c_char_p,
                                      C.c_char_p, C.c_int, C.c_double]),
    ("dare_system_create", C.c_int, [_P, C.POINTER(_P)]),
    ("dare_system_destroy", C.c_int, [_P]),
    ("dare_system_set_bc", C.c_int, [_P, C.c_int, C.c_int, C.c_double]),
    ("dare_assemble", C.c_int, [_P, C.POINTER(AssemblyDesc), _P]),
    ("dare_system_set_bc_component", C.c_int, [_P, C.c_int, C.c_int, C.c_int, C.c_double]),
    ("dare_assemble_terms", C.c_int, [_P, C.POINTER(TermDesc), C.c_int, _P]),
    ("dare_system_set_coefficients", C.c_int, [_P, _P, _P, _P]),
    ("dare_system_get_coefficients", C.c_int, [_P, _P, _P]),
    ("dare_system_set_initial_guess", C.c_int, [_P, _P]),
    ("dare_system_get_solution", C.c_int, [_P, _P]),
    ("dare_system_device_ptr", _P, [_P, C.c_int]),
    ("dare_system_csr_nnz", C.c_int64, [_P]),
    ("dare_system_export_csr", C.c_int, [_P, _P, _P, _P]),
    ("dare_system_copy_to", C.c_int, [_P, _P]),
    ("dare_solver_params_default", None, [C.POINTER(SolverParams)]),
    ("dare_bicgstab2_solve", C.c_int, [_P, C.POINTER(SolverParams), C.POINTER(SolveReport)]),
    ("dare_timestep", C.c_int, [_P, _P, C.POINTER(AssemblyDesc), C.POINTER(SolverParams),
                                C.POINTER(SolveReport)]),
    ("dare_timesteps_host", C.c_int, [_P, _P, C.POINTER(AssemblyDesc), C.POINTER(SolverParams), C.c_int, _P,
                                      C.POINTER(SolveReport)]),
    ("dare_face_average", C.c_int, [_P, _P, C.POINTER(_P)]),
    ("dare_slabs_create", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(_P)]),
    ("dare_slabs_destroy", C.c_int, [_P]),
    ("dare_slabs_count", C.c_int, [_P]),
    ("dare_slabs_range", C.c_int, [_P, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("dare_slabs_system", _P, [_P, C.c_int]),
    ("dare_slabs_field", _P, [_P, C.c_int]),
    ("dare_slabs_set_bc", C.c_int, [_P, C.c_int, C.c_int, C.c_double]),
    ("dare_slabs_scatter", C.c_int, [_P, _P]),
    ("dare_slabs_gather", C.c_int, [_P, _P]),
    ("dare_slabs_exchange_halo", C.c_int, [_P]),
    ("dare_slabs_copy_to_old", C.c_int, [_P]),
    ("dare_slabs_assemble", C.c_int, [_P, C.POINTER(AssemblyDesc)]),
    ("dare_slabs_solve", C.c_int, [_P, C.POINTER(SolverParams), C.POINTER(SolveReport)]),
    ("dare_slabs_copy_to", C.c_int, [_P]),
    ("dare_slabs_timestep", C.c_int, [_P, C.POINTER(AssemblyDesc), C.POINTER(SolverParams),
                                      C.POINTER(SolveReport)]),
    ("dare_residual_norm_noalloc", C.c_int, [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int), _P, _P, _P, _P,
                                             _P, C.c_char_p, C.c_int]),
    ("dare_batch_create", C.c_int, [_P, C.c_int, _P, C.POINTER(_P)]),
    ("dare_batch_destroy", C.c_int, [_P]),
    ("dare_batch_num_cells", C.c_int64, [_P, C.c_int]),
    ("dare_batch_set_field", C.c_int, [_P, C.c_int, _P]),
    ("dare_batch_get_field", C.c_int, [_P, C.c_int, _P]),
    ("dare_batch_zero_fields", C.c_int, [_P]),
    ("dare_batch_solve", C.c_int, [_P, _P, _P]),
    ("dare_batch_autotune", C.c_int, [_P, _P, C.POINTER(C.c_int)]),
    ("dare_batch_get_tuning", C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
]


class UNetTrainParams(C.Structure):
    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float),
                ("batch", C.c_int), ("steps", C.c_int), ("max_pairs_per_rhs", C.c_int), ("seed", C.c_uint64)]


class UNetTrainReport(C.Structure):
    _fields_ = [("pairs_added", C.c_int), ("pairs_total", C.c_int), ("plain_iters", C.c_int), ("steps", C.c_int),
                ("loss_first", C.c_double), ("loss_last", C.c_double)]


class LearnedParams(C.Structure):
    _fields_ = [("iteration_budget", C.c_int), ("inner_max_it", C.c_int), ("inner_rel_tol", C.c_double),
                ("max_refinements", C.c_int)]


_SIGS += [
    ("dare_unet_train_params_default", None, [C.POINTER(UNetTrainParams)]),
    ("dare_learned_params_default", None, [C.POINTER(LearnedParams)]),
    ("dare_unet_create", C.c_int, [_P, C.POINTER(C.c_int), C.c_uint64, C.POINTER(_P)]),
    ("dare_unet_create_coarse", C.c_int, [_P, C.POINTER(C.c_int), C.c_uint64, C.POINTER(_P)]),
    ("dare_unet_set_wait_limit", C.c_int, [_P, C.c_int64]),
    ("dare_unet_debug_skip_plane", C.c_int, [_P]),
    ("dare_unet_system_shape", C.c_int, [_P, C.POINTER(C.c_int)]),
    ("dare_unet_destroy", C.c_int, [_P]),
    ("dare_unet_num_params", C.c_int64, [_P]),
    ("dare_unet_get_weights", C.c_int, [_P, _P, C.c_int64]),
    ("dare_unet_set_weights", C.c_int, [_P, _P, C.c_int64]),
    ("dare_unet_apply", C.c_int, [_P, _P, _P]),
    ("dare_unet_loss_grad", C.c_int, [_P, _P, _P, C.c_int, C.POINTER(C.c_double), _P]),
    ("dare_unet_train_step", C.c_int, [_P, _P, _P, C.c_int, C.POINTER(UNetTrainParams), C.POINTER(C.c_double)]),
    ("dare_unet_train_on_system", C.c_int, [_P, _P, C.c_double, C.POINTER(UNetTrainParams),
                                            C.POINTER(UNetTrainReport)]),
    ("dare_unet_stats", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("dare_unet_read_activation", C.c_int, [_P, C.c_int, _P, C.c_int64]),
    ("dare_unet_launch_info", C.c_int, [_P, C.c_int, C.c_int, C.POINTER(C.c_int64)]),
    ("dare_bicgstab2_learned", C.c_int, [_P, _P, C.POINTER(SolverParams), C.POINTER(LearnedParams),
                                         C.POINTER(SolveReport)]),
]


class BatchInstance(C.Structure):
    _fields_ = [("n", C.c_int64 * 3), ("size", C.c_double * 3), ("D", C.c_double), ("dt", C.c_double),
                ("bc_type", C.c_int * 6), ("bc_value", C.c_double * 6)]


class BatchReport(C.Structure):
    _fields_ = [("iters", C.c_int), ("converged", C.c_int), ("status", C.c_int), ("breakdown_step", C.c_int),
                ("res_abs", C.c_double), ("b_norm", C.c_double), ("tol_abs", C.c_double)]

_lib = None


def library_path() -> str:
    return LIB_PATH


def lib():
    """Load libdare_gpu.so (fails loudly: there is no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"dare_b200: {LIB_PATH} is missing; build it with `python -m dare_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class DareError(RuntimeError):
    pass


def _destroy(fn_name: str, h) -> None:
    """Release a handle from a finalizer.  At interpreter shutdown the module's
    globals may already be gone, and the process is ending anyway: skip."""
    try:
        getattr(_lib, fn_name)(h)
    except Exception:
        pass


def _check(rc: int, ctx=None, what: str = ""):
    if rc != 0:
        msg = lib().dare_ctx_last_error(ctx).decode() if ctx else ""
        raise DareError(f"{what} failed with status {rc}: {msg}")


def _ptr(a: np.ndarray):
    if a is None:
        return None
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data_as(C.c_void_p)


class Context:
    """One device and one CUDA stream (dare_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().dare_ctx_create(device, C.byref(h))
        if rc != 0:
            raise DareError(f"dare_ctx_create(device={device}) failed with status {rc}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().dare_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        _check(lib().dare_ctx_synchronize(self.h), self.h, "synchronize")

    def set_stream(self, stream_ptr: int | None):
        _check(lib().dare_ctx_set_stream(self.h, stream_ptr), self.h, "set_stream")

    @property
    def stream(self) -> int:
        return lib().dare_ctx_get_stream(self.h) or 0

    @property
    def launch_count(self) -> int:
        return int(lib().dare_ctx_launch_count(self.h))

    def set_profiling(self, on: bool):
        _check(lib().dare_ctx_set_profiling(self.h, int(on)), self.h, "set_profiling")

    def reset_kernel_stats(self):
        lib().dare_ctx_reset_kernel_stats(self.h)

    def timer_start(self):
        _check(lib().dare_ctx_timer_start(self.h), self.h, "timer_start")

    def timer_stop(self) -> float:
        ms = C.c_double()
        _check(lib().dare_ctx_timer_stop(self.h, C.byref(ms)), self.h, "timer_stop")
        return ms.value

    def kernel_stats(self, name: str):
        ms = C.c_double()
        n = C.c_int64()
        _check(lib().dare_ctx_kernel_stats(self.h, KERNEL_IDS[name], C.byref(ms), C.byref(n)), self.h, "stats")
        return ms.value, n.value


class Grid:
    """Cartesian grid on one rank (Grid::Cartesian<Dim> + CartesianRepresentation)."""

    def __init__(self, ctx: Context, n, size=None, num_ghost: int = 2, periodic=None, staggered=None):
        """``n`` and ``size`` describe the (base) grid; ``staggered`` (one flag
        per direction) selects a staggered representation: one more cell
        along each staggered, non-periodic direction, shifted by half a cell."""
        dim = len(n)
        self.ctx = ctx
        nn = (C.c_int64 * 3)(*(list(n) + [1] * (3 - dim)))
        sz = list(size) if size is not None else [1.0] * dim
        ss = (C.c_double * 3)(*(sz + [1.0] * (3 - dim)))
        pp_ = list(periodic) if periodic is not None else [0] * dim
        pp = (C.c_int * 3)(*([int(x) for x in pp_] + [0] * (3 - dim)))
        h = C.c_void_p()
        if staggered is None:
            _check(lib().dare_grid_create(ctx.h, dim, nn, ss, num_ghost, pp, C.byref(h)), ctx.h, "grid_create")
        else:
            st = (C.c_int * 3)(*([int(x) for x in staggered] + [0] * (3 - dim)))
            _check(lib().dare_grid_create_staggered(ctx.h, dim, nn, ss, num_ghost, pp, st, C.byref(h)), ctx.h,
                   "grid_create")
        self.h = h
        info = GridInfo()
        lib().dare_grid_get_info(h, C.byref(info))
        self.info = info
        self.dim = dim
        self.n = tuple(int(info.n[d]) for d in range(3))
        self.ghosted_shape = tuple(int(info.n_ghosted[d]) for d in range(3))
        self.num_cells = int(info.num_cells)
        self.num_cells_ghosted = int(info.num_cells_ghosted)

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None):
            _destroy("dare_grid_destroy", self.h)
            self.h = None

    @property
    def dx(self):
        return [self.info.dx[d] for d in range(3)]

    @property
    def origin(self):
        return [self.info.origin[d] for d in range(3)]

    @property
    def volume(self):
        return self.info.volume

    @property
    def area(self):
        return [self.info.area[d] for d in range(3)]

    def face_shape(self, d: int):
        s = list(self.n)
        s[d] += 1
        return tuple(s)


class Field:
    """Time levels of ghosted grid vectors on the device (Data::Field<Grid,SC,N>).

    Host arrays interleave the components: ghosted[cell * N + c]."""

    def __init__(self, grid: Grid, num_levels: int = 2, components: int = 1):
        self.grid = grid
        h = C.c_void_p()
        _check(lib().dare_field_create_n(grid.h, num_levels, components, C.byref(h)), grid.ctx.h, "field_create")
        self.h = h
        self.num_levels = num_levels
        self.components = components

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None):
            _destroy("dare_field_destroy", self.h)
            self.h = None

    def upload(self, values: np.ndarray, level: int = 0):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if a.size != self.grid.num_cells_ghosted * self.components:
            raise ValueError("field upload expects the ghosted layout")
        _check(lib().dare_field_upload(self.h, level, _ptr(a)), self.grid.ctx.h, "field_upload")

    def download(self, level: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Copy a level to the host; `out` (e.g. pinned memory) is filled in place when given."""
        size = self.grid.num_cells_ghosted * self.components
        a = np.empty(size, dtype=np.float64) if out is None else out.reshape(-1)
        if a.size != size or a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("field download expects a contiguous float64 ghosted buffer")
        _check(lib().dare_field_download(self.h, level, _ptr(a)), self.grid.ctx.h, "field_download")
        return a

    def device_ptr(self, level: int = 0) -> int:
        return lib().dare_field_device_ptr(self.h, level)

    def exchange_halo(self):
        _check(lib().dare_field_exchange_halo(self.h), self.grid.ctx.h, "exchange_halo")

    def copy_to_old(self):
        _check(lib().dare_field_copy_to_old(self.h), self.grid.ctx.h, "copy_to_old")


class DeviceArray:
    """A plain device buffer owned by a torch tensor (plumbing for face arrays)."""

    def __init__(self, host: np.ndarray | None, device: int = 0):
        import torch
        self.t = None if host is None else torch.from_numpy(
            np.ascontiguousarray(host, dtype=np.float64)).to(f"cuda:{device}")

    @classmethod
    def from_tensor(cls, t) -> "DeviceArray":
        a = cls(None)
        a.t = t.contiguous()
        return a

    @property
    def ptr(self) -> int:
        return self.t.data_ptr()


@dataclass
class Assembly:
    """Descriptor of the fused per-cell functor (see dare_assembly_desc)."""
    dt: float = 0.0
    D: float | None = None
    face_D: tuple | None = None        # 3 device pointers (int) or DeviceArray
    vel: tuple | None = None           # constant velocity
    face_vel: tuple | None = None      # 3 device pointers (int) or DeviceArray
    limiter: str = "VANLEER"
    scheme: str = "EULER_BACKWARD"     # time scheme of the div(...) terms (SCHEME)

    def to_c(self) -> AssemblyDesc:
        a = AssemblyDesc()
        a.dt = self.dt
        if self.face_D is not None:
            a.diffusion = 2
            for d, p in enumerate(self.face_D):
                a.face_D[d] = p.ptr if isinstance(p, DeviceArray) else p
        elif self.D is not None:
            a.diffusion = 1
            a.D = float(self.D)
        if self.face_vel is not None:
            a.convection = 2
            for d, p in enumerate(self.face_vel):
                a.face_vel[d] = p.ptr if isinstance(p, DeviceArray) else p
        elif self.vel is not None:
            a.convection = 1
            for d, v in enumerate(self.vel):
                a.vel[d] = float(v)
        a.limiter = LIMITER[self.limiter]
        a.scheme = SCHEME[self.scheme]
        return a



TERM_KINDS = {"DDT": 0, "DIFFUSION": 1, "CONVECTION": 2, "COEFFS": 3}
TERM_OPS = {"SET": 0, "ADD": 1, "SUB": 2}


@dataclass
class Term:
    """One MatrixBlock expression of a composed functor (see dare_term):
    ``Term("DDT", "SET", dt=dt)`` is ``mb = ddt(field)``, ``Term("DIFFUSION",
    "SUB")`` is ``mb -= div(grad(mb))``, ``Term("CONVECTION", "ADD", component=0,
    vel=(u, v, 0))`` is ``mb.Add(0, div(TVD(u) * field).GetSlice(0))``;
    ``Term("COEFFS", "ADD", coef=(c, None, ...), rhs=b)`` adds per-cell slot
    and right-hand-side values the caller computed on the device (device
    pointers or DeviceArray, one component's cells each)."""
    kind: str
    op: str = "ADD"
    component: int = -1
    dt: float = 0.0
    D: float = 1.0
    face_D: tuple | None = None
    vel: tuple | None = None
    face_vel: tuple | None = None
    limiter: str = "VANLEER"
    scheme: str = "EULER_BACKWARD"
    coef: tuple | None = None          # COEFFS: 7 slot arrays (None entries: 0)
    rhs: object = None                 # COEFFS: right-hand-side array

    def to_c(self) -> TermDesc:
        t = TermDesc()
        t.kind = TERM_KINDS[self.kind.upper()]
        t.op = TERM_OPS[self.op.upper()]
        t.component = int(self.component)
        t.dt = float(self.dt)
        t.D = float(self.D)
        if self.face_D is not None:
            for d, p in enumerate(self.face_D):
                t.face_D[d] = p.ptr if isinstance(p, DeviceArray) else p
        if self.vel is not None:
            for d, v in enumerate(self.vel):
                t.vel[d] = float(v)
        if self.face_vel is not None:
            for d, p in enumerate(self.face_vel):
                t.face_vel[d] = p.ptr if isinstance(p, DeviceArray) else p
        t.limiter = LIMITER[self.limiter]
        t.scheme = SCHEME[self.scheme]
        if self.coef is not None:
            for q, p in enumerate(self.coef):
                t.coef[q] = p.ptr if isinstance(p, DeviceArray) else p
        if self.rhs is not None:
            t.coef_rhs = self.rhs.ptr if isinstance(self.rhs, DeviceArray) else self.rhs
        return t


class MatrixSystem:
    """Structured 7-diagonal system A x = B (Matrix::Trilinos<SC>); with N
    components one stencil per component, rows and columns cell * N + c."""

    def __init__(self, grid: Grid, components: int = 1):
        self.grid = grid
        h = C.c_void_p()
        _check(lib().dare_system_create_n(grid.h, components, C.byref(h)), grid.ctx.h, "system_create")
        self.h = h
        self.components = components
        self.rows = grid.num_cells * components

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None) and getattr(self, "_owned", True):
            _destroy("dare_system_destroy", self.h)
        self.h = None

    def set_bc(self, face: int, kind: int, value: float = 0.0, component: int = -1):
        """Condition of a face, for every component or for one."""
        if component < 0:
            _check(lib().dare_system_set_bc(self.h, face, kind, value), self.grid.ctx.h, "set_bc")
        else:
            _check(lib().dare_system_set_bc_component(self.h, component, face, kind, value), self.grid.ctx.h,
                   "set_bc_component")

    def build(self, field: Field, assembly):
        """Trilinos<SC>::Build; x0 = field level 0.  ``assembly`` is the fused
        functor (an Assembly) or a composed one (a sequence of Term)."""
        if isinstance(assembly, Assembly):
            desc = assembly.to_c()
            _check(lib().dare_assemble(self.h, C.byref(desc), field.h), self.grid.ctx.h, "assemble")
            return
        terms = list(assembly)
        arr = (TermDesc * max(1, len(terms)))()
        for i, t in enumerate(terms):
            arr[i] = t.to_c()
        _check(lib().dare_assemble_terms(self.h, arr, len(terms), field.h), self.grid.ctx.h, "assemble_terms")

    def set_coefficients(self, diag: np.ndarray | None, rhs: np.ndarray | None = None, x0: np.ndarray | None = None):
        d = None if diag is None else np.ascontiguousarray(diag, dtype=np.float64)
        r = None if rhs is None else np.ascontiguousarray(rhs, dtype=np.float64)
        x = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        _check(lib().dare_system_set_coefficients(self.h, _ptr(d), _ptr(r), _ptr(x)), self.grid.ctx.h, "set_coef")

    def coefficients(self):
        n = self.rows
        diag = np.empty((7, n), dtype=np.float64)
        rhs = np.empty(n, dtype=np.float64)
        _check(lib().dare_system_get_coefficients(self.h, _ptr(diag), _ptr(rhs)), self.grid.ctx.h, "get_coef")
        return diag, rhs

    def solution(self) -> np.ndarray:
        x = np.empty(self.rows, dtype=np.float64)
        _check(lib().dare_system_get_solution(self.h, _ptr(x)), self.grid.ctx.h, "get_solution")
        return x

    def set_initial_guess(self, x0: np.ndarray):
        self.set_coefficients(None, None, x0)

    def device_ptr(self, which: int) -> int:
        return lib().dare_system_device_ptr(self.h, which)

    def export_csr(self):
        nnz = int(lib().dare_system_csr_nnz(self.h))
        n = self.rows
        rowptr = np.empty(n + 1, dtype=np.int64)
        cols = np.empty(nnz, dtype=np.int64)
        vals = np.empty(nnz, dtype=np.float64)
        _check(lib().dare_system_export_csr(self.h, _ptr(rowptr), _ptr(cols), _ptr(vals)), self.grid.ctx.h, "csr")
        return rowptr, cols, vals

    def copy_to(self, field: Field):
        _check(lib().dare_system_copy_to(self.h, field.h), self.grid.ctx.h, "copy_to")


class BiCGStab2:
    """BiCGStab(2) with the reference's parameter names (Matrix::BiCGStab2)."""

    def __init__(self, params: dict | None = None, precond: str = "JACOBI", precision: str = "FP64"):
        p = SolverParams()
        lib().dare_solver_params_default(C.byref(p))
        params = params or {}
        if "Convergence Tolerance" in params:
            p.tol = float(params["Convergence Tolerance"])
        if "Maximum Iterations" in params:
            p.max_it = int(params["Maximum Iterations"])
        p.precond = {"NONE": PREC_NONE, "JACOBI": PREC_JACOBI}[precond.upper()]
        p.precision = {"FP64": PRECISION_FP64, "FP32_REFINE": PRECISION_FP32_REFINE}[precision.upper()]
        for k, v in params.items():
            if hasattr(p, k):
                setattr(p, k, v)
        self.params = p
        self.report = None

    def solve(self, system: MatrixSystem) -> dict:
        rep = SolveReport()
        _check(lib().dare_bicgstab2_solve(system.h, C.byref(self.params), C.byref(rep)), system.grid.ctx.h,
               "bicgstab2_solve")
        self.report = rep.as_dict()
        return self.report

    def get_num_iters(self) -> int:
        return self.report["iters"] if self.report else 0


class Slabs:
    """The grid of ``system`` split into slabs of i-planes on its device: the
    reference's distribution over ranks (CartesianDistribution.h:94-380)
    with its halo exchange (HaloBuffer.inl:30-208) and a sum over all slabs
    in every dot product of the solve.  Slab s owns planes ``ranges[s]`` with
    its own field, rows and solver vectors; boundary planes cross to the x
    neighbours before every assembly (num_ghost planes of the field) and
    every SpMV (one plane of the operand), for every field component.  FP64."""

    def __init__(self, system: MatrixSystem, num_slabs: int, num_levels: int = 2):
        self.ctx = system.grid.ctx
        self.grid = system.grid
        self.components = system.components
        h = C.c_void_p()
        _check(lib().dare_slabs_create(system.h, num_slabs, num_levels, C.byref(h)), self.ctx.h, "slabs_create")
        self.h = h
        self.count = int(lib().dare_slabs_count(h))
        self.ranges = []
        for s in range(self.count):
            a, b = C.c_int64(), C.c_int64()
            _check(lib().dare_slabs_range(h, s, C.byref(a), C.byref(b)), self.ctx.h, "slabs_range")
            self.ranges.append((a.value, b.value))
        self.periodic_x = bool(self.grid.info.periodic[0])

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None):
            _destroy("dare_slabs_destroy", self.h)
            self.h = None

    def system(self, s: int) -> MatrixSystem:
        """Slab s's rows as a MatrixSystem view (coefficients, solution)."""
        v = MatrixSystem.__new__(MatrixSystem)
        v._owned = False
        v.h = C.c_void_p(lib().dare_slabs_system(self.h, s))
        v.grid = self.grid
        v.components = self.components
        i0, i1 = self.ranges[s]
        v.rows = (i1 - i0) * self.grid.n[1] * self.grid.n[2] * self.components
        return v

    def field_ptr(self, s: int, level: int = 0) -> int:
        return lib().dare_field_device_ptr(lib().dare_slabs_field(self.h, s), level)

    def set_bc(self, face: int, kind: int, value: float = 0.0):
        _check(lib().dare_slabs_set_bc(self.h, face, kind, value), self.ctx.h, "slabs_set_bc")

    def scatter(self, field: Field):
        _check(lib().dare_slabs_scatter(self.h, field.h), self.ctx.h, "slabs_scatter")

    def gather(self, field: Field):
        _check(lib().dare_slabs_gather(self.h, field.h), self.ctx.h, "slabs_gather")

    def exchange_halo(self):
        _check(lib().dare_slabs_exchange_halo(self.h), self.ctx.h, "slabs_exchange_halo")

    def copy_to_old(self):
        _check(lib().dare_slabs_copy_to_old(self.h), self.ctx.h, "slabs_copy_to_old")

    def copy_to(self):
        _check(lib().dare_slabs_copy_to(self.h), self.ctx.h, "slabs_copy_to")

    def face_slices(self, faces):
        """Each slab's part of the three face arrays of the grid (host arrays
        of shapes n + e_d): x faces i0 .. i1 (face 0 after the last plane on
        a periodic x), the slab's planes of the y and z faces."""
        n0 = self.grid.n[0]
        out = []
        for i0, i1 in self.ranges:
            fx = np.asarray(faces[0])
            if self.periodic_x and i1 == n0:
                fx = np.concatenate([fx[i0:n0], fx[0:1]])
            else:
                fx = fx[i0:i1 + 1]
            out.append((np.ascontiguousarray(fx),) +
                       tuple(np.ascontiguousarray(np.asarray(f)[i0:i1]) for f in faces[1:]))
        return out

    def _descs(self, assemblies):
        assemblies = list(assemblies)
        if len(assemblies) != self.count:
            raise ValueError("one Assembly per slab")
        arr = (AssemblyDesc * self.count)()
        for s, a in enumerate(assemblies):
            arr[s] = a.to_c()
        return arr

    def assemble(self, assemblies):
        """Trilinos::Build on every slab (one Assembly per slab, its face
        arrays from face_slices)."""
        _check(lib().dare_slabs_assemble(self.h, self._descs(assemblies)), self.ctx.h, "slabs_assemble")

    def solve(self, solver: "BiCGStab2") -> dict:
        rep = SolveReport()
        _check(lib().dare_slabs_solve(self.h, C.byref(solver.params), C.byref(rep)), self.ctx.h, "slabs_solve")
        solver.report = rep.as_dict()
        return solver.report

    def timestep(self, assemblies, solver: "BiCGStab2") -> dict:
        rep = SolveReport()
        _check(lib().dare_slabs_timestep(self.h, self._descs(assemblies), C.byref(solver.params), C.byref(rep)),
               self.ctx.h, "slabs_timestep")
        solver.report = rep.as_dict()
        return solver.report

    def solution(self) -> np.ndarray:
        """The slabs' solutions in the grid's cell order."""
        return np.concatenate([self.system(s).solution() for s in range(self.count)])


def timestep(system: MatrixSystem, field: Field, assembly: Assembly, solver: BiCGStab2) -> dict:
    """Build, Solve, CopyTo, ExchangeHaloCells, CopyDataVectorsToOldTimeStep on the device."""
    desc = assembly.to_c()
    rep = SolveReport()
    _check(lib().dare_timestep(system.h, field.h, C.byref(desc), C.byref(solver.params), C.byref(rep)),
           system.grid.ctx.h, "timestep")
    solver.report = rep.as_dict()
    return solver.report


def timesteps_host(system: MatrixSystem, field: Field, assembly: Assembly, solver: BiCGStab2, steps: int,
                   host: np.ndarray) -> list:
    """`steps` implicit steps of a field kept in host memory (``host``: pinned,
    the field's device layout, float64): each step reads its input from
    ``host`` and writes its result back, the result of one step travelling
    down while the input of the next travels up."""
    size = field.grid.num_cells_ghosted * field.components
    if host.size != size or host.dtype != np.float64 or not host.flags["C_CONTIGUOUS"]:
        raise ValueError("timesteps_host expects a contiguous float64 buffer of the field's ghosted size")
    desc = assembly.to_c()
    reps = (SolveReport * steps)()
    _check(lib().dare_timesteps_host(system.h, field.h, C.byref(desc), C.byref(solver.params), steps, _ptr(host),
                                     reps), system.grid.ctx.h, "timesteps_host")
    out = [r.as_dict() for r in reps]
    solver.report = out[-1]
    return out


def write_vtk(fields, names, base_path: str, grid_name: str, step: int, time: float = -1.0, level: int = 0):
    """io::VTKWriter(exman, time, step).Write(base_path, &vec...) for fields of one
    grid: <base_path>/<grid_name>_<step>.pvts plus its piece in the subdirectory
    <grid_name>_<step>/ (the ghosted grid, one Float64 cell array per field)."""
    fields = list(fields)
    names = [str(n) for n in names]
    if len(fields) != len(names) or not fields:
        raise ValueError("write_vtk: one name per field")
    hs = (_P * len(fields))(*[f.h for f in fields])
    ns = (C.c_char_p * len(names))(*[n.encode() for n in names])
    ctx = fields[0].grid.ctx.h
    _check(lib().dare_vtk_write(hs, level, ns, len(fields), base_path.encode(), grid_name.encode(), step, time),
           ctx, "vtk_write")


def write_vtk_host(n, size, num_ghost: int, arrays, names, base_path: str, grid_name: str, step: int,
                   time: float = -1.0):
    """The same writer from host arrays over the ghosted grid (no GPU involved)."""
    dim = len(n)
    n3 = (C.c_int64 * 3)(*(list(n) + [1] * (3 - dim)))
    s3 = (C.c_double * 3)(*(list(size) + [1.0] * (3 - dim)))
    arrays = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in arrays]
    ps = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    ns = (C.c_char_p * len(names))(*[str(x).encode() for x in names])
    _check(lib().dare_vtk_write_host(dim, n3, s3, num_ghost, ps, ns, len(arrays), base_path.encode(),
                                     grid_name.encode(), step, time), None, "vtk_write_host")


def face_average(grid: Grid, cell_D_ptr: int, face_ptrs) -> None:
    arr = (C.c_void_p * 3)(*[p.ptr if isinstance(p, DeviceArray) else p for p in face_ptrs])
    _check(lib().dare_face_average(grid.h, cell_D_ptr, arr), grid.ctx.h, "face_average")


class Batch:
    """Many independent implicit diffusion steps solved in one persistent launch.

    ``instances``: dicts with ``n`` (3 ints), ``size`` (3 floats), ``D``, ``dt``,
    ``bc`` = {face: (kind, value)} for faces WEST..TOP (Dirichlet/Neumann).
    """

    def __init__(self, ctx: Context, instances):
        self.ctx = ctx
        arr = (BatchInstance * len(instances))()
        for q, ins in enumerate(instances):
            a = arr[q]
            for d in range(3):
                a.n[d] = int(ins["n"][d])
                a.size[d] = float(ins.get("size", (1.0, 1.0, 1.0))[d])
            a.D = float(ins["D"])
            a.dt = float(ins["dt"])
            for face in range(1, 7):
                kind, val = ins["bc"].get(face, (BC_NEUMANN, 0.0))
                a.bc_type[face - 1] = kind
                a.bc_value[face - 1] = val
        h = C.c_void_p()
        _check(lib().dare_batch_create(ctx.h, len(instances), arr, C.byref(h)), ctx.h, "batch_create")
        self.h = h
        self.count = len(instances)

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None):
            _destroy("dare_batch_destroy", self.h)
            self.h = None

    def num_cells(self, idx: int) -> int:
        return int(lib().dare_batch_num_cells(self.h, idx))

    def set_field(self, idx: int, values: np.ndarray):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        if a.size != self.num_cells(idx):
            raise ValueError("batch field size")
        _check(lib().dare_batch_set_field(self.h, idx, _ptr(a)), self.ctx.h, "batch_set_field")

    def get_field(self, idx: int) -> np.ndarray:
        a = np.empty(self.num_cells(idx), dtype=np.float64)
        _check(lib().dare_batch_get_field(self.h, idx, _ptr(a)), self.ctx.h, "batch_get_field")
        return a

    def zero_fields(self):
        _check(lib().dare_batch_zero_fields(self.h), self.ctx.h, "batch_zero_fields")

    def solve(self, solver: "BiCGStab2", reports: bool = True):
        rep = (BatchReport * self.count)() if reports else None
        _check(lib().dare_batch_solve(self.h, C.byref(solver.params), rep), self.ctx.h, "batch_solve")
        if not reports:
            return None
        return [{"iters": r.iters, "converged": bool(r.converged), "status": SOLVE_STATUS.get(r.status, r.status),
                 "breakdown_step": r.breakdown_step, "res_abs": r.res_abs, "b_norm": r.b_norm, "tol_abs": r.tol_abs}
                for r in rep]

    def autotune(self, solver: "BiCGStab2") -> dict:
        blk = C.c_int()
        _check(lib().dare_batch_autotune(self.h, C.byref(solver.params), C.byref(blk)), self.ctx.h, "autotune")
        vec = (C.c_int * 8)()
        lib().dare_batch_get_tuning(self.h, C.byref(blk), vec)
        return {"block": blk.value, "cells_per_thread_by_size": list(vec)}


class LearnedPreconditioner:
    """The linear conv U-Net preconditioner of the Jacobi-folded system
    (dare_unet): 8 bias-free 3x3x3 convolutions over 4 levels, BF16 weights,
    FP32 tensor-core accumulation, trained on the GPU.  ``coarse=False``:
    N(u) = u + U(u) on the system's grid ``n``; ``coarse=True``: the
    coarse-correction form N(u) = u + P U(R u), the network on the 2x
    restricted grid n / 2 (``net_shape``)."""

    LAYERS = (("enc0", 0, 1, 16), ("enc1", 1, 16, 32), ("enc2", 2, 32, 64), ("enc3", 3, 64, 64),
              ("dec3", 3, 64, 64), ("dec2", 2, 64, 32), ("dec1", 1, 32, 16), ("dec0", 0, 16, 1))
    ACTIVATIONS = (("S0", 0, 16), ("P1", 1, 16), ("S1", 1, 32), ("P2", 2, 32), ("S2", 2, 64), ("P3", 3, 64),
                   ("E3", 3, 64))

    def __init__(self, ctx: Context, n, seed: int = 0, coarse: bool = False):
        self.ctx = ctx
        self.n = tuple(int(x) for x in n)
        self.coarse = bool(coarse)
        nn = (C.c_int * 3)(*self.n)
        h = C.c_void_p()
        create = lib().dare_unet_create_coarse if coarse else lib().dare_unet_create
        _check(create(ctx.h, nn, C.c_uint64(seed), C.byref(h)), ctx.h, "unet_create")
        self.h = h
        self.num_params = int(lib().dare_unet_num_params(h))
        self.num_cells = self.n[0] * self.n[1] * self.n[2]
        # the grid the convolutions (and the training pairs) live on
        self.net_shape = tuple(x // 2 for x in self.n) if coarse else self.n
        self.net_cells = int(np.prod(self.net_shape))

    def __del__(self, _destroy=_destroy):
        if getattr(self, "h", None):
            _destroy("dare_unet_destroy", self.h)
            self.h = None

    @staticmethod
    def train_params(**kw) -> UNetTrainParams:
        p = UNetTrainParams()
        lib().dare_unet_train_params_default(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def set_wait_limit(self, polls: int = 0):
        """Polls of the convolutions' role-to-role waits (0: the default)."""
        _check(lib().dare_unet_set_wait_limit(self.h, int(polls)), self.ctx.h, "unet_set_wait_limit")

    def debug_skip_plane(self):
        """Test hook: the next forward convolution's first CTA leaves one plane unstaged."""
        _check(lib().dare_unet_debug_skip_plane(self.h), self.ctx.h, "unet_debug_skip_plane")

    def get_weights(self) -> np.ndarray:
        w = np.empty(self.num_params, dtype=np.float32)
        _check(lib().dare_unet_get_weights(self.h, _ptr(w), self.num_params), self.ctx.h, "unet_get_weights")
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().dare_unet_set_weights(self.h, _ptr(w), w.size), self.ctx.h, "unet_set_weights")

    def apply(self, u_ptr: int, z_ptr: int):
        """z = N(u) for FP32 device vectors (raw pointers)."""
        _check(lib().dare_unet_apply(self.h, u_ptr, z_ptr), self.ctx.h, "unet_apply")

    def activation(self, which: int) -> np.ndarray:
        _, lev, ch = self.ACTIVATIONS[which]
        cells = int(np.prod([x >> lev for x in self.net_shape]))
        a = np.empty(cells * ch, dtype=np.float32)
        _check(lib().dare_unet_read_activation(self.h, which, _ptr(a), a.size), self.ctx.h, "unet_read_activation")
        return a.reshape(cells, ch)

    def loss_grad(self, r_ptr: int, e_ptr: int, count: int, want_grad: bool = True):
        loss = C.c_double()
        g = np.empty(self.num_params, dtype=np.float32) if want_grad else None
        _check(lib().dare_unet_loss_grad(self.h, r_ptr, e_ptr, count, C.byref(loss), _ptr(g)), self.ctx.h,
               "unet_loss_grad")
        return loss.value, g

    def train_step(self, r_ptr: int, e_ptr: int, count: int, params: UNetTrainParams | None = None) -> float:
        p = params or self.train_params()
        loss = C.c_double()
        _check(lib().dare_unet_train_step(self.h, r_ptr, e_ptr, count, C.byref(p), C.byref(loss)), self.ctx.h,
               "unet_train_step")
        return loss.value

    def train_on_system(self, system: MatrixSystem, tol: float, params: UNetTrainParams | None = None) -> dict:
        p = params or self.train_params()
        rep = UNetTrainReport()
        _check(lib().dare_unet_train_on_system(self.h, system.h, tol, C.byref(p), C.byref(rep)), self.ctx.h,
               "unet_train_on_system")
        return {name: getattr(rep, name) for name, _ in rep._fields_}

    def launch_info(self, layer: int, kind: int = 0) -> dict | None:
        """Launch shape of a convolution kernel (kind 0 forward, 1 data
        gradient, 2 weight gradient) after its first launch."""
        v = (C.c_int64 * 8)()
        if lib().dare_unet_launch_info(self.h, layer, kind, v) != 0:
            return None
        keys = ("grid_x", "grid_y", "grid_z", "smem", "planes_per_cta", "taps_or_ring", "tmem_cols", "ctas_per_sm")
        return dict(zip(keys, list(v)))

    def stats(self) -> dict:
        s, q = C.c_int64(), C.c_int64()
        lib().dare_unet_stats(self.h, C.byref(s), C.byref(q))
        return {"steps": s.value, "pairs_seen": q.value}

    @staticmethod
    def learned_params(**kw) -> LearnedParams:
        p = LearnedParams()
        lib().dare_learned_params_default(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p

    def solve(self, system: MatrixSystem, solver: BiCGStab2, params: LearnedParams | None = None) -> dict:
        """Learned-preconditioned mixed-precision BiCGStab2 with the automatic
        fallback to the plain FP64 Jacobi-BiCGStab2."""
        lp = params or self.learned_params()
        rep = SolveReport()
        _check(lib().dare_bicgstab2_learned(system.h, self.h, C.byref(solver.params), C.byref(lp), C.byref(rep)),
               system.grid.ctx.h, "bicgstab2_learned")
        solver.report = rep.as_dict()
        return solver.report
