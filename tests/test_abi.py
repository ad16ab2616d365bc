"""The C ABI library loads and exports every function include/*.h declares
(no compute: runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from common import ROOT

from diff_solver_b200 import _native


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:XsStatus|size_t|uint64_t|int|const char\*|void)\s+(xs_[a-z0-9_]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_python_signatures_cover_the_header():
    assert declared_functions() <= set(_native.SIGNATURES), set(declared_functions()) - set(_native.SIGNATURES)


STRUCTS = ["XsGrid", "XsScalarBoundary", "XsVelocityBoundary", "XsPressureSolve", "XsSolveStats", "XsInflow", "XsCollider",
           "XsSmokeModel", "XsState", "XsControl", "XsParameters", "XsStepCache"]


def test_struct_layouts_match_header(tmp_path):
    """sizeof and every field offset of the ctypes mirrors equal what the C
    compiler makes of include/diff_smoke.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or "/usr/bin/gcc"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "diff_smoke.h"', "int main(void) {"]
    for name in STRUCTS:
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in getattr(_native, name)._fields_:
            lines.append(f'printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include", str(src), "-o", str(exe)], check=True)
    want = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for name in STRUCTS:
        cls = getattr(_native, name)
        assert ctypes.sizeof(cls) == int(want[name]), name
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == int(want[f"{name}.{field}"]), (name, field)


def test_status_strings_and_launch_counter_without_gpu():
    lib = _native.lib()
    assert lib.xs_status_string(_native.XS_NOT_CONVERGED).decode().startswith("pressure")
    assert isinstance(lib.xs_launch_count(), int)


def test_workspace_queries_without_gpu():
    lib = _native.lib()
    g = _native.XsGrid(16, 14, 12, 1 / 16, 1 / 32)
    n = 16 * 14 * 12
    ws = lib.xs_projection_workspace_bytes(g)
    assert ws >= n * (8 + 4 * 5)
    bad = _native.XsGrid(0, 14, 12, 1 / 16, 1 / 32)
    assert lib.xs_projection_workspace_bytes(bad) == 0
    m = _native.XsSmokeModel()
    m.grid = g
    fwd = lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0)
    diff = lib.xs_smoke_workspace_bytes(ctypes.byref(m), 1)
    assert diff > fwd > ws


@pytest.mark.parametrize("extents", [(2**32 - 1, 4, 4), (4, 2**32 - 1, 4), (2**22, 2**22, 2**22), (2**16, 2**16, 2),
                                     (1024, 1024, 4096)])
def test_grids_past_32_bit_indexing_are_rejected(extents):
    # kernels index with 32 bits: (nx + 1)(ny + 1)(nz + 1) must stay below
    # 2^32, without the extent sum or the product wrapping around
    lib = _native.lib()
    g = _native.XsGrid(*extents, 1e-3, 5e-4)
    assert lib.xs_projection_workspace_bytes(g) == 0
    assert lib.xs_source_forward(None, g, None, None, None, None, 0, 0, None) == _native.XS_INVALID_ARGUMENT


def test_largest_grids_within_32_bit_indexing_are_accepted():
    lib = _native.lib()
    # 1023 x 1023 x 4094: (nx + 1)(ny + 1)(nz + 1) = 2^32 - 2^20
    assert lib.xs_projection_workspace_bytes(_native.XsGrid(1023, 1023, 4094, 1e-3, 5e-4)) > 0
    assert lib.xs_projection_workspace_bytes(_native.XsGrid(512, 512, 256, 1 / 512, 1 / 1024)) > 0


def test_warm_start_options_are_validated_without_gpu():
    """The ring (0..5 solutions) and the coarse-grid correction (a factor that
    divides the grid, with a ring and no colliders) size the workspace; other
    settings make the model invalid (0 bytes)."""
    lib = _native.lib()
    m = _native.XsSmokeModel()
    m.grid = _native.XsGrid(32, 32, 16, 1 / 32, 1 / 64)
    base = lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0)
    m.warm_start_history = 5
    ring = lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0)
    assert ring > base
    m.warm_start_coarsening = 4
    coarse = lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0)
    assert coarse > ring
    m.warm_start_coarsening = 3  # does not divide 32
    assert lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0) == 0
    m.warm_start_coarsening = 32  # 16 / 32 is not whole
    assert lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0) == 0
    m.warm_start_coarsening = 2
    m.warm_start_history = 0  # no ring
    assert lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0) == 0
    m.warm_start_history = 6
    m.warm_start_coarsening = 0
    assert lib.xs_smoke_workspace_bytes(ctypes.byref(m), 0) == 0


def test_invalid_arguments_are_rejected_before_any_launch():
    lib = _native.lib()
    g = _native.XsGrid(0, 4, 4, 0.25, 0.1)
    st = lib.xs_source_forward(None, g, None, None, None, None, 0, 0, None)
    assert st == _native.XS_INVALID_ARGUMENT
    solve = _native.XsPressureSolve(0, 10, 1e-6, None)
    g2 = _native.XsGrid(4, 4, 4, 0.25, 0.1)
    assert lib.xs_pressure_solve(None, g2, ctypes.byref(solve), 0, None, _native.XsScalarBoundary(), None, None, None) == \
        _native.XS_INVALID_ARGUMENT
