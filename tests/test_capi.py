"""The C-ABI shared library loads and exports every entry point that
include/pigfem_b200.h declares (no compute calls: no GPU needed)."""
import ctypes
import os
import re

import pytest

from helpers import gpu_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "pigfem_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(pg_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    from pigfem_assignment_b200._lib import LIB_PATH, DECLARED_SYMBOLS
    lib = ctypes.CDLL(LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(DECLARED_SYMBOLS) == syms


def test_version_and_error_strings():
    from pigfem_assignment_b200._lib import lib
    assert b"sm_100a" in lib.pg_version()
    assert lib.pg_last_error() is not None


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_ctx_create_without_gpu_fails_loudly():
    import pigfem_assignment_b200.problem as pb
    from pigfem_assignment_b200._lib import PgError
    from pigfem_assignment_b200.rve import RVE
    m = pb.Mesh(RVE(nx=4, ny=4, inclusions=[(0.5, 0.5, 0.25, 1)]))
    with pytest.raises(PgError) as ei:
        pb.DeviceContext(m)
    assert ei.value.code == 3  # PG_ERR_CUDA: no CPU fallback


def test_null_arguments_return_status():
    from pigfem_assignment_b200._lib import lib
    assert lib.pg_mesh_build(None, None) == 1
    assert lib.pg_assemble_linear(None, None) == 1
    assert lib.pg_solve_linear(None, None, None) == 1
