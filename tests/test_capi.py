"""CPU tests of the C-ABI library: it loads without a GPU, exports every
symbol the header declares, its structs match the header's layout, and it
fails loudly (no CPU fallback) when no device is present."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "aether_fluid.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(afl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import aether_fluid
    lib = aether_fluid.load()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {n for n, _, _ in aether_fluid._lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_struct_layout_matches_header(tmp_path):
    """sizeof/offsetof seen by a C compiler equal the ctypes mirror's."""
    from aether_fluid import _lib
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "aether_fluid.h"
int main(void) {
  printf("%zu %zu %zu\n", sizeof(afl_params), sizeof(afl_telemetry), sizeof(afl_solve_info));
  printf("%zu %zu %zu %zu\n", offsetof(afl_params, sphere_center),
         offsetof(afl_params, mixed_inner_rel_tol), offsetof(afl_params, reserved_f64),
         offsetof(afl_solve_info, initial_residual));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o",
                           str(exe)])
    lines = subprocess.check_output([str(exe)]).decode().split("\n")
    sizes = [int(x) for x in lines[0].split()]
    offs = [int(x) for x in lines[1].split()]
    assert sizes == [ctypes.sizeof(_lib.AflParams), ctypes.sizeof(_lib.AflTelemetry),
                     ctypes.sizeof(_lib.AflSolveInfo)]
    assert offs == [_lib.AflParams.sphere_center.offset,
                    _lib.AflParams.mixed_inner_rel_tol.offset,
                    _lib.AflParams.reserved_f64.offset,
                    _lib.AflSolveInfo.initial_residual.offset]


def test_defaults_are_the_reference_defaults():
    """src/fluid.rs:79-83 and the SOR constant of :398."""
    from aether_fluid import _lib
    p = _lib.default_params()
    assert (p.vorticity_eps, p.buoyancy_beta, p.gravity_alpha) == (5.5, 6.8, 0.45)
    assert (p.solver_kind, p.solver_iters) == (0, 32)
    assert p.sor_omega == 1.65 and p.cg_rel_tol == 0.0
    assert p.source_kind == 0 and p.precision == 0


def test_invalid_grid_rejected_before_device_use():
    """src/fluid.rs:54 asserts n >= 6; the ABI returns INVALID_ARGUMENT."""
    from aether_fluid import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.afl_create(5, 8, 8, None, ctypes.byref(h)) == 1
    assert b">= 6" in lib.afl_last_error()
    assert lib.afl_destroy(None) == 0
    assert lib.afl_step(None, 0.1, 0.0, None, None) == 1


def test_invalid_params_rejected():
    from aether_fluid import _lib
    lib = _lib.load()
    p = _lib.default_params()
    p.solver_kind = 7
    h = ctypes.c_void_p()
    assert lib.afl_create(8, 8, 8, ctypes.byref(p), ctypes.byref(h)) == 1
    assert b"solver_kind" in lib.afl_last_error()


@pytest.mark.skipif(gpu_available(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    import aether_fluid
    with pytest.raises(aether_fluid.AetherFluidError) as e:
        aether_fluid.FluidSolver3D(8, 8, 8)
    assert e.value.status == 2  # AFL_ERR_CUDA, never a CPU fallback


def test_product_does_not_reference_oracle():
    """The product sources never load, link or call the oracle."""
    pkg = os.path.join(ROOT, "aether-core-engine_b200")
    for dirpath, _, files in os.walk(pkg):
        if "_build" in dirpath:
            continue
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                text = open(os.path.join(dirpath, f)).read()
                for bad in ("liboracle", "ofl_", "import oracle", "from oracle",
                            "fluid_oracle"):
                    assert bad not in text, (f, bad)
