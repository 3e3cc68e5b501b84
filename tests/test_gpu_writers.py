"""The VTK and cohesive-openings writers against the files the reference's own
writers (Writer_ASCII_VTK, WriterCohesiveOpenings) made of the same state
(golden fixtures, oracle/ref_driver.cpp).

The state is the reference's: its solution (and, for the cohesive mesh, its
committed delta_max before the last step, from which the last residual
assembly forms the reactions).  Structure -- headers, counts, connectivity,
cell types, material numbers -- must match token for token.  Values are
printed as floats with six significant digits (the CSV at sixteen): a value
may differ in its last printed digit where the device's FP64 rounding lands
on the other side of a float, so numbers compare within 2e-6 of the larger
of the value and its section's scale (1e-12 for the CSV)."""
import math

import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from helpers import golden, rve_from_golden

pytestmark = pytest.mark.gpu


class _Holder:
    def __init__(self, ctx):
        self.ctx = ctx


def _sections(text):
    out, name = {}, "header"
    for line in text.splitlines():
        if not line.strip():
            continue
        head = line.split()[0]
        if head in ("POINTS", "CELLS", "CELL_TYPES", "POINT_DATA", "CELL_DATA", "VECTORS", "SCALARS"):
            name = " ".join(line.split()[:2])
            out.setdefault(name, []).append(line.split())
            continue
        out.setdefault(name, []).append(line.split())
    return out


def _num(tok):
    try:
        return float(tok)
    except ValueError:
        return None


def compare_vtk(got, ref, rtol=2e-6):
    a, b = _sections(got), _sections(ref)
    assert list(a) == list(b)
    for name in b:
        la, lb = a[name], b[name]
        assert len(la) == len(lb), name
        vals = [abs(v) for row in lb for v in map(_num, row) if v is not None and math.isfinite(v)]
        scale = max(vals) if vals else 0.0
        for ra, rb in zip(la, lb):
            assert len(ra) == len(rb), (name, ra, rb)
            for ta, tb in zip(ra, rb):
                if ta == tb:
                    continue
                va, vb = _num(ta), _num(tb)
                assert va is not None and vb is not None, (name, ta, tb)
                if math.isnan(vb):
                    assert math.isnan(va), (name, ta, tb)
                    continue
                assert abs(va - vb) <= rtol * max(abs(vb), scale), (name, ta, tb)


@pytest.mark.parametrize("name", ["linear_8x8.npz", "linear_3inc.npz", "linear_cfg0.npz"])
def test_vtk_matches_reference_writer(name, tmp_path):
    g = golden(name)
    m = pb.Mesh(rve_from_golden(g))
    e = m.export()
    ctx = pb.DeviceContext(m)
    ctx.set_vector(0, np.concatenate([g["U.f"], g["U.p"]])[e["ref_dof"]])
    path = tmp_path / "out.vtk"
    pb.Writer_ASCII_VTK(_Holder(ctx)).write(str(path), 1.0)
    compare_vtk(path.read_text(), bytes(g["vtk.text"]).decode())
    ctx.close()


def _cohesive_final_state():
    g = golden("cohesive_16x16.npz")
    rve = rve_from_golden(g, cohesive=True)
    n = int(g["cfg.nsteps"][0])
    rve.strain = float(g["cfg.strain_per_step"][0]) * n
    m = pb.Mesh(rve)
    e = m.export()
    ctx = pb.DeviceContext(m)
    ctx.set_vector(0, np.concatenate([g[f"step{n}.U.f"], g[f"step{n}.U.p"]])[e["ref_dof"]])
    ctx.set_isv(g[f"step{n - 1}.isv.delta_max"], committed=True)
    pb.Assembler(ctx).assemble_nonlinear(float(g["cfg.dt"][0]), True, False)
    return g, e, ctx


def test_cohesive_vtk_matches_reference_writer(tmp_path):
    g, e, ctx = _cohesive_final_state()
    # the reactions the writer prints are the reference's P_int on prescribed DOFs
    F = ctx.vector(1)
    Fr = np.empty_like(F)
    Fr[e["ref_dof"]] = F
    pint_p = g["Pint.p"]
    nf = int(g["dof.n_free"][0])
    np.testing.assert_allclose(Fr[nf:], pint_p, rtol=1e-8, atol=1e-8 * np.abs(pint_p).max())
    path = tmp_path / "out.vtk"
    pb.Writer_ASCII_VTK(_Holder(ctx)).write(str(path), 0.4)
    compare_vtk(path.read_text(), bytes(g["vtk.text"]).decode())
    ctx.close()


def test_cohesive_openings_match_reference_writer(tmp_path):
    g, _, ctx = _cohesive_final_state()
    path = tmp_path / "openings.csv"
    pb.WriterCohesiveOpenings(_Holder(ctx)).write(str(path))
    got = [l.split(",") for l in path.read_text().splitlines()]
    ref = [l.split(",") for l in bytes(g["openings.text"]).decode().splitlines()]
    assert len(got) == len(ref) and len(ref) > 0
    A = np.array([[float(v) for v in r] for r in got])
    B = np.array([[float(v) for v in r] for r in ref])
    np.testing.assert_array_equal(A[:, 0], B[:, 0])
    np.testing.assert_allclose(A[:, 1:], B[:, 1:], rtol=1e-10, atol=1e-10 * np.abs(B[:, 1:]).max())
    ctx.close()


def test_openings_writer_refuses_a_mesh_without_interface(tmp_path):
    from pigfem_assignment_b200 import _lib
    m = pb.Mesh(rve_from_golden(golden("linear_8x8.npz")))
    ctx = pb.DeviceContext(m)
    with pytest.raises(_lib.PgError) as ei:
        pb.WriterCohesiveOpenings(_Holder(ctx)).write(str(tmp_path / "x.csv"))
    assert ei.value.code == _lib.PG_ERR_ARG
    ctx.close()
