"""CPU checks of the C ABI: the library loads and exports every symbol the
headers under include/ declare; argument validation needs no device."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^DARE_API\s+[\w\s\*]+?\b(dare_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def gpu_lib():
    import dare_b200
    return dare_b200.lib()


def test_headers_declare_symbols():
    assert len(declared_symbols()) >= 30


def test_library_exports_every_declared_symbol(gpu_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", os.path.join(ROOT, "dare_b200", "libdare_gpu.so")],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(dare_\w+)$", out, flags=re.M))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        getattr(gpu_lib, s)


def test_python_binding_covers_header():
    import dare_b200
    bound = {name for name, _, _ in dare_b200._SIGS}
    assert set(declared_symbols()) <= bound


def test_null_arguments_rejected_without_device(gpu_lib):
    # argument validation happens before any CUDA call
    assert gpu_lib.dare_ctx_create(0, None) != 0
    assert gpu_lib.dare_grid_destroy(None) == 0
    assert gpu_lib.dare_field_exchange_halo(None) != 0
    assert gpu_lib.dare_system_set_bc(None, 1, 1, 0.0) != 0
    assert gpu_lib.dare_bicgstab2_solve(None, None, None) != 0
    # the slab path and the host-resident loop check their handles first too
    assert gpu_lib.dare_slabs_create(None, 2, 2, None) != 0
    assert gpu_lib.dare_slabs_destroy(None) != 0
    assert gpu_lib.dare_slabs_count(None) < 0
    assert gpu_lib.dare_slabs_system(None, 0) is None
    assert gpu_lib.dare_slabs_field(None, 0) is None
    assert gpu_lib.dare_slabs_scatter(None, None) != 0
    assert gpu_lib.dare_slabs_exchange_halo(None) != 0
    assert gpu_lib.dare_slabs_assemble(None, None) != 0
    assert gpu_lib.dare_slabs_solve(None, None, None) != 0
    assert gpu_lib.dare_slabs_set_bc(None, 1, 1, 0.0) != 0
    assert gpu_lib.dare_timesteps_host(None, None, None, None, 1, None, None) != 0


def test_solver_defaults_match_reference():
    import dare_b200
    p = dare_b200.SolverParams()
    dare_b200.lib().dare_solver_params_default(C.byref(p))
    # BiCGStab2 constructor defaults: tol 1e-8, max 100 (BiCGStab2.inl:29-31)
    assert p.tol == 1e-8 and p.max_it == 100 and p.precond == dare_b200.PREC_JACOBI


def test_cxx_header_compiles(tmp_path):
    src = tmp_path / "t.cpp"
    src.write_text('#include "dare_gpu.hpp"\nint main() { dare_b200::BiCGStab2 s({{"Maximum Iterations", 7}});'
                   ' (void)sizeof(dare_b200::Slabs); return s.Params().max_it == 7 ? 0 : 1; }\n')
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                    str(src)], check=True)


def test_no_product_import_of_oracle():
    # the product package never imports the CPU checker
    for f in glob.glob(os.path.join(ROOT, "dare_b200", "**", "*.py"), recursive=True):
        assert "oracle" not in open(f).read().replace("no CPU fallback", ""), f
