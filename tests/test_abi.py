"""The C-ABI library and the C++ layer, without a GPU: every function declared in
include/mpcd_c.h is exported by libmpcd_b200.so, the Python struct mirrors have the C sizes,
the C++ shim compiles standalone, and the drivers reject a wrong command line."""
import ctypes as C
import os
import re
import shutil
import subprocess

import pytest

from src_incompressible_openmp_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "mpcd_c.h")
LIB = os.path.join(ROOT, "src_incompressible_openmp_b200", "libmpcd_b200.so")


def declared_functions():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(mpcd_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_phase_api():
    names = declared_functions()
    for f in ("mpcd_ctx_create", "mpcd_set_state", "mpcd_apply_bc", "mpcd_srd_shift_cells", "mpcd_srd_collide",
              "mpcd_cell_fields", "mpcd_zone_pass", "mpcd_liquid_closure", "mpcd_step", "mpcd_cell_fields_static"):
        assert f in names, f


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIB):
        pytest.fail("libmpcd_b200.so not built (run __graft_entry__.build())")
    lib = C.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_struct_mirrors_match_c(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    structs = ["mpcd_params_c", "mpcd_wallinfo_c", "mpcd_pass_metrics_c", "mpcd_closure_metrics_c",
               "mpcd_cellfields_c", "mpcd_closure_detail_c", "mpcd_step_metrics_c"]
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "mpcd_c.h"\nint main(void){\n' +
                   "".join(f'printf("%zu\\n", sizeof({s}));\n' for s in structs) + "return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run([gcc, "-I", os.path.dirname(HDR), "-o", str(exe), str(src)], check=True)
    sizes = [int(s) for s in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    mirrors = [_abi.ParamsC, _abi.WallInfoC, _abi.PassMetricsC, _abi.ClosureMetricsC, _abi.CellFieldsC,
               _abi.ClosureDetailC, _abi.StepMetricsC]
    for name, size, m in zip(structs, sizes, mirrors):
        assert C.sizeof(m) == size, (name, C.sizeof(m), size)


def test_cpp_shim_compiles_standalone(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "use.cpp"
    src.write_text('#include "types.h"\n#include "zone_pass_openmp.h"\n#include "liquid_closure.h"\n'
                   "int main(){ mpcd::Params p{}; p.boundary_left = \"periodic\"; p.boundary_right = \"periodic\";\n"
                   "return mpcd::is_periodic_pair(p, \"x\") ? 0 : 1; }\n")
    subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include", "compat"),
                    "-I", os.path.join(ROOT, "include"), str(src)], check=True)


@pytest.mark.parametrize("exe", ["src_incompressible_openmp_b200/bin/mpcd_bench", "oracle/_ref/ref_main_b200"])
def test_drivers_reject_wrong_command_line(exe):
    path = os.path.join(ROOT, exe)
    if not os.path.exists(path):
        pytest.fail(f"not built: {path}")
    r = subprocess.run([path, "only-one-arg"], capture_output=True, text=True)
    assert r.returncode == 2 and "Usage" in r.stderr


def test_status_on_cpu_only_host():
    """Without a GPU the library loads and says so; nothing falls back to the CPU."""
    from src_incompressible_openmp_b200 import native
    if native.device_available():
        pytest.skip("a GPU is present")
    from src_incompressible_openmp_b200.cases import poiseuille_params
    with pytest.raises(native.MpcdError):
        native.Context(poiseuille_params(8, 8, 2))
