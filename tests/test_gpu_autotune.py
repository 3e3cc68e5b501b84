"""Assembly launch shapes: every shape the autotuner may pick assembles the
same K (against the oracle), and the autotuner times them all and keeps the
fastest."""
import ctypes as C

import numpy as np
import pytest

import oracle
import pigfem_assignment_b200.problem as pb
from helpers import bsr_to_csr, rel_fro
from pigfem_assignment_b200 import _lib
from pigfem_assignment_b200.rve import RVE, config0

pytestmark = pytest.mark.gpu


def gpu_K(ctx, e):
    return bsr_to_csr(e["row_ptr"], e["col"], ctx.matrix_values())


@pytest.mark.parametrize("tile", [32, 64, 128, 256])
@pytest.mark.parametrize("persistent", [0, 1])
@pytest.mark.parametrize("warps", [2, 4, 8])
def test_every_launch_shape_assembles_the_same_K(tile, persistent, warps):
    # two inclusions close together give cut elements of several size classes
    rve = RVE(nx=40, ny=40, inclusions=[(0.3, 0.5, 0.2, 1), (0.72, 0.5, 0.2, 1)], strain=0.01)
    m = pb.Mesh(rve)
    e = m.export()
    ctx = pb.DeviceContext(m)
    _lib.check(_lib.lib.pg_ctx_set_tuning(ctx.handle, tile, persistent, warps))
    pb.Assembler(ctx).assemble_linear()
    Ko, _, _ = oracle.from_product(e, pb.template_table(), rve).assemble()
    assert rel_fro(gpu_K(ctx, e), Ko) <= 1e-12
    ctx.close()


@pytest.mark.parametrize("tile", [32, 64, 128, 256])
@pytest.mark.parametrize("persistent", [0, 1])
@pytest.mark.parametrize("warps", [2, 8])
def test_every_launch_shape_assembles_the_same_tangent_and_residual(tile, persistent, warps):
    # the residual and tangent passes of a cohesive mesh (bilinear law, damaged
    # state) through every launch shape: K and f_int against the oracle
    rve = RVE(nx=20, ny=20, inclusions=[(0.45, 0.5, 0.27, 1)], cohesive=True, coh_law=1,
              coh_params=(30.0, 0.01, 1.0e6, 1.0, 200.0), strain=0.02)
    m = pb.Mesh(rve)
    e = m.export()
    ctx = pb.DeviceContext(m)
    _lib.check(_lib.lib.pg_ctx_set_tuning(ctx.handle, tile, persistent, warps))
    rng = np.random.default_rng(5)
    U = 1e-4 * rng.standard_normal(m.info["n_dof"])
    isv_c = np.abs(2e-5 * rng.standard_normal(m.info["n_cohesive_qp"]))
    ctx.set_vector(0, U)
    ctx.set_isv(isv_c, committed=True)
    om = oracle.from_product(e, pb.template_table(), rve)
    Ko, fo, io = om.assemble(u=U, dt=0.02, isv_c=isv_c, want_K=True, want_f=True)
    asm = pb.Assembler(ctx)
    asm.assemble_nonlinear(0.02, False, True)   # tangent pass
    assert rel_fro(gpu_K(ctx, e), Ko) <= 1e-12
    asm.assemble_nonlinear(0.02, True, False)   # residual pass
    assert np.linalg.norm(ctx.vector(1) - fo) / np.linalg.norm(fo) <= 1e-12
    np.testing.assert_allclose(ctx.isv(committed=False), io, rtol=1e-13, atol=0)
    ctx.close()


def test_autotune_times_every_shape_and_keeps_the_fastest():
    rve = config0()
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    ms_tri = (C.c_float * 5)()
    ms_cut = (C.c_float * 3)()
    _lib.check(_lib.lib.pg_ctx_autotune(prob.ctx.handle, 3, ms_tri, ms_cut))
    assert all(v > 0 for v in ms_tri) and all(v > 0 for v in ms_cut)
    tile, pers, warps = C.c_int32(), C.c_int32(), C.c_int32()
    _lib.check(_lib.lib.pg_ctx_tuning(prob.ctx.handle, C.byref(tile), C.byref(pers), C.byref(warps)))
    best_tri = int(np.argmin(list(ms_tri)))
    if best_tri == 4:
        assert tile.value in (128, 256)  # threads per CTA of the structured-grid kernel
    else:
        assert (tile.value, pers.value) == ((32, 64)[best_tri // 2], best_tri % 2)
    assert warps.value == (2, 4, 8)[int(np.argmin(list(ms_cut)))]
    # the tuned context still solves to the reference tolerance
    st = prob.solve_problem()
    assert st.status == 0
    prob.ctx.close()


@pytest.mark.parametrize("tile", [128, 256])
def test_pipelined_grid_kernel_writes_the_same_bits(tile):
    # the persistent kernel stages the next tile asynchronously, and the cut
    # kernels may run beside it on a second stream; the values are the same
    # arithmetic on the same inputs: identical K and f
    from pigfem_assignment_b200.rve import config1, scaled
    rve = scaled(config1(), 256)
    m = pb.Mesh(rve)
    ctx = pb.DeviceContext(m)
    rng = np.random.default_rng(7)
    ctx.set_vector(0, 1e-3 * rng.standard_normal(m.info["n_dof"]))
    out = []
    for persistent, overlap in ((0, 0), (0, 1), (1, 0), (1, 1), (1, 2)):
        _lib.check(_lib.lib.pg_ctx_set_tuning(ctx.handle, tile, persistent, 4))
        _lib.check(_lib.lib.pg_ctx_cut_overlap(ctx.handle, overlap, None))
        pb.Assembler(ctx).assemble_nonlinear(1.0, True, True)
        out.append((ctx.matrix_values(), ctx.vector(1)))
    for k in range(1, len(out)):
        assert np.array_equal(out[0][0], out[k][0])
        assert np.array_equal(out[0][1], out[k][1])
    ctx.close()
