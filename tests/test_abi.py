"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: these run without a GPU)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared_functions() -> list[str]:
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(p2c_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def libpath():
    from p2cccd_b200 import build

    if not build.LIB.exists():
        build.build()
    return build.LIB


def test_headers_declare_entry_points():
    names = _declared_functions()
    assert "p2c_certify_pt_batch" in names and "p2c_last_error" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol(libpath):
    lib = ctypes.CDLL(str(libpath))
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_every_declared_symbol():
    from p2cccd_b200 import _lib

    missing = [n for n in _declared_functions() if n not in _lib.SIGNATURES]
    assert not missing, f"declared but not bound in p2cccd_b200._lib: {missing}"


def test_host_only_entry_points_answer_without_gpu(libpath):
    from p2cccd_b200 import _lib

    lib = _lib.load()
    assert lib.p2c_abi_version() >= 1
    assert lib.p2c_is_cuda_exact_built() == 1
    assert lib.p2c_certify_workspace_bytes(1000) >= 64


def test_record_layouts_match_header():
    from p2cccd_b200 import records

    assert records.POINT_TRIANGLE_DTYPE.itemsize == 240
    assert records.EDGE_EDGE_DTYPE.itemsize == 240
    assert records.INTERVAL_RESULT_DTYPE.itemsize == 72
    assert records.INTERVAL_RESULT_DTYPE.fields["toi_upper"][1] == 24
    assert records.INTERVAL_RESULT_DTYPE.fields["reason_code"][1] == 64
    import oracle

    assert oracle.RESULT == records.INTERVAL_RESULT_DTYPE
    assert oracle.PT.itemsize == 240 and oracle.EE.itemsize == 240
    rec = np.zeros(1, dtype=records.POINT_TRIANGLE_DTYPE)
    assert rec.dtype.fields["triangle_v2"][1] == 16 + 3 * 56


def test_serving_struct_layouts_match_header(tmp_path):
    """The Python mirror's ctypes / numpy layouts of the serving structs
    equal the C header's (sizes and offsets printed by a C compiler)."""
    import shutil
    import subprocess

    from p2cccd_b200 import serve

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stddef.h>
#include <stdio.h>
#include "p2c_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\\n", sizeof(p2c_serve_config), sizeof(p2c_serve_mesh), sizeof(p2c_serve_request),
         sizeof(p2c_serve_result), sizeof(p2c_serve_stats));
  printf("%zu %zu %zu %zu\\n", offsetof(p2c_serve_result, latency_ms), offsetof(p2c_serve_result, certify),
         offsetof(p2c_serve_result, anyhit), offsetof(p2c_serve_config, cert));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = [int(v) for v in out]
    assert sizes[:5] == [ctypes.sizeof(serve.ServeConfigC), ctypes.sizeof(serve.ServeMeshC),
                         ctypes.sizeof(serve.ServeRequestC), serve.SERVE_RESULT_DTYPE.itemsize,
                         serve.SERVE_STATS_DTYPE.itemsize]
    f = serve.SERVE_RESULT_DTYPE.fields
    assert sizes[5:8] == [f["latency_ms"][1], f["certify"][1], f["anyhit"][1]]
    assert sizes[8] == serve.ServeConfigC.cert.offset


def test_reference_checker_libraries_load():
    """Every checker library under oracle/_ref resolves all its symbols (a
    missing one would only show on the GPU box otherwise)."""
    import oracle

    for so in (oracle.REF_SO, oracle.REF_TOOL_SO, oracle.REF_CUDA_SO):
        if so.exists():
            ctypes.CDLL(str(so))
