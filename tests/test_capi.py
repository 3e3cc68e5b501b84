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


def header_struct_fields(name):
    """Field names, in order, of `typedef struct name { ... } name;` in the header."""
    txt = open(os.path.join(ROOT, "include", "pigfem_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    m = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), txt, flags=re.S)
    assert m, name
    out = []
    for decl in m.group(1).split(";"):
        decl = decl.strip()
        if not decl:
            continue
        # "type a, b, *c[5]": the names follow the type's last word
        decl = re.sub(r"\[[^\]]*\]", "", decl)
        head, _, rest = decl.partition(",")
        names = [head.split()[-1]] + [r.strip() for r in rest.split(",") if r.strip()] if rest else [head.split()[-1]]
        out += [n.lstrip("*") for n in names]
    return out


@pytest.mark.parametrize("cname, pyname", [("pg_rve_desc", "RveDesc"), ("pg_mesh_info", "MeshInfo"),
                                           ("pg_solver_cfg", "SolverCfg"), ("pg_solve_stats", "SolveStats"),
                                           ("pg_newton_cfg", "NewtonCfg"), ("pg_step_stats", "StepStats"),
                                           ("pg_pred_history", "PredHistory")])
def test_binding_structs_follow_the_header(cname, pyname):
    """The ctypes mirrors have the header's fields in the header's order (a
    field added in C and not in Python shifts every later one)."""
    from pigfem_assignment_b200 import _lib
    assert [f[0] for f in getattr(_lib, pyname)._fields_] == header_struct_fields(cname)


@pytest.mark.parametrize("fn, pyname", [("pg_solver_cfg_default", "SolverCfg"), ("pg_newton_cfg_default", "NewtonCfg")])
def test_config_defaults_write_inside_the_struct(fn, pyname):
    """The default writers fill exactly the struct the binding allocates:
    the bytes after it stay untouched, and the last field (deterministic)
    reads back as its default."""
    from pigfem_assignment_b200 import _lib
    T = getattr(_lib, pyname)
    size = ctypes.sizeof(T)
    buf = (ctypes.c_uint8 * (size + 64))(*([0xAB] * (size + 64)))
    getattr(_lib.lib, fn)(ctypes.cast(buf, ctypes.POINTER(T)))
    assert bytes(buf[size:]) == b"\xab" * 64
    cfg = T.from_buffer(buf)
    assert cfg.deterministic == 1
