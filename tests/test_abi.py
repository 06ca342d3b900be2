"""The C-ABI library: builds, loads, exports what include/pstm_cuda.h declares,
and the ctypes mirror matches the header's struct layouts (CPU only; no
compute call needs a GPU here)."""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pstm_cuda.h")


@pytest.fixture(scope="module")
def lib_path():
    from pstm_b200 import build
    return build.build()


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pstm_cuda_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported_and_bound(lib_path):
    from pstm_b200 import _native as nat
    L = ctypes.CDLL(lib_path)
    names = declared_functions()
    assert names, "no declarations found"
    for n in names:
        assert hasattr(L, n), f"{n} declared but not exported"
        assert n in nat.SIGNATURES, f"{n} declared but not bound in _native.SIGNATURES"
    assert set(nat.SIGNATURES) <= set(names)


def test_library_loads_and_reports_abi(lib_path):
    from pstm_b200 import _native as nat
    L = nat.load()
    assert L.pstm_cuda_abi_version() == nat.ABI_VERSION
    src = open(HEADER).read()
    assert f"#define PSTM_CUDA_ABI_VERSION {nat.ABI_VERSION}" in src


def test_null_context_errors_without_gpu(lib_path):
    """Calls on a NULL context fail with NOT_INITIALIZED, like the reference's
    RuntimeError("Kernel not initialized") (numba_cpu_optimized.py:555-556)."""
    from pstm_b200 import _native as nat
    L = nat.load()
    rc = L.pstm_cuda_synchronize(None)
    assert rc == nat.ERR_NOT_INITIALIZED
    assert b"not initialized" in L.pstm_cuda_last_error(None)
    rc = L.pstm_cuda_migrate_tile_host(None, None, None, None, None)
    assert rc == nat.ERR_NOT_INITIALIZED
    assert L.pstm_cuda_migrate_bins_dev(None, None, None, None, None, None, 0, None) == nat.ERR_NOT_INITIALIZED
    assert L.pstm_cuda_autotune_bins(None, None, None, None, None, None, 0, 0, None) == nat.ERR_NOT_INITIALIZED
    assert L.pstm_cuda_surrogate_param_count() == 8897
    assert L.pstm_cuda_surrogate_samples(None, None, 0, 0, 0, None, None, None, None) == nat.ERR_NOT_INITIALIZED
    assert L.pstm_cuda_surrogate_eval(None, None, None, 0, None, None) == nat.ERR_NOT_INITIALIZED
    assert L.pstm_cuda_migrate_tile_learned_dev(None, None, None, None, None, None, 0.0, 0, None,
                                                None) == nat.ERR_NOT_INITIALIZED
    with pytest.raises(RuntimeError, match="not initialized"):
        nat.check(rc, None, L)


def _c_layout(tmp_path):
    """sizeof/offsetof of every descriptor field, from the C compiler."""
    from pstm_b200 import _native as nat
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "pstm_cuda.h"', 'int main(void){']
    for cname, cls in (("pstm_traces_desc", nat.TracesDesc), ("pstm_output_desc", nat.OutputDesc),
                       ("pstm_velocity_desc", nat.VelocityDesc), ("pstm_params", nat.Params),
                       ("pstm_bin_desc", nat.BinDesc), ("pstm_tune_result", nat.TuneResult),
                       ("pstm_surrogate_domain", nat.SurrogateDomain), ("pstm_surrogate", nat.Surrogate),
                       ("pstm_learned_report", nat.LearnedReport)):
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


def test_ctypes_structs_match_header_layout(tmp_path):
    from pstm_b200 import _native as nat
    lay = _c_layout(tmp_path)
    for cname, cls in (("pstm_traces_desc", nat.TracesDesc), ("pstm_output_desc", nat.OutputDesc),
                       ("pstm_velocity_desc", nat.VelocityDesc), ("pstm_params", nat.Params),
                       ("pstm_bin_desc", nat.BinDesc), ("pstm_tune_result", nat.TuneResult),
                       ("pstm_surrogate_domain", nat.SurrogateDomain), ("pstm_surrogate", nat.Surrogate),
                       ("pstm_learned_report", nat.LearnedReport)):
        assert lay[(cname, "size")] == ctypes.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert lay[(cname, f)] == getattr(cls, f).offset, (cname, f)
