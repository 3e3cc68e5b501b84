"""Stress and strain recovery (Problem::compute_stress_strain,
src/Problem.cpp:428-534) and the homogenised response on the GPU.

Against the reference run on the same meshes (golden fixtures made by
oracle/ref_driver.cpp): with the reference's own solution loaded, every
volumetric quadrature point's strain, stress and J W, in the reference's
point order.  The reference's points of a collapsed integration child have
zero weight and NaN strain (its inverse map is singular there); the device
marks the same points NaN.  At full size, through a property that holds for
any continuous field whose x-displacement is prescribed on the left and right
edges: the volume average of the strain xx equals the applied strain.

Tolerances: J W within 1e-11 of the point's weight or of the largest weight
(a cut child's Jacobian is formed from its corner coordinates by a different
but equivalent expression, whose rounding on a small child reaches ~1e-11 of
the element's size); strain and stress 1e-10
of the field's largest magnitude (gradients of small cut children are large,
and the reference forms them through its own inverse map); averages 1e-12."""
import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from helpers import golden, rve_from_golden
from pigfem_assignment_b200.rve import config1

pytestmark = pytest.mark.gpu

GOLDEN = ["linear_8x8.npz", "linear_cfg0.npz", "linear_3inc.npz"]


def _with_reference_solution(name):
    g = golden(name)
    rve = rve_from_golden(g)
    m = pb.Mesh(rve)
    e = m.export()
    ctx = pb.DeviceContext(m)
    uref = np.concatenate([g["U.f"], g["U.p"]])
    ctx.set_vector(0, uref[e["ref_dof"]])
    return g, ctx


@pytest.mark.parametrize("name", GOLDEN)
def test_points_match_reference(name):
    g, ctx = _with_reference_solution(name)
    pts, off, mean = ctx.compute_stress_strain()
    # the same number of volumetric points per element, in the same order
    np.testing.assert_array_equal(np.diff(off), g["qp.count"])
    n = pts.shape[0]
    assert n == g["qp.jw"].size
    eps_r = g["qp.strain"].reshape(n, 3)
    sig_r = g["qp.stress"].reshape(n, 3)
    jw_r = g["qp.jw"]
    np.testing.assert_allclose(pts[:, 6], jw_r, rtol=1e-11, atol=1e-11 * np.abs(jw_r).max())
    # collapsed children: zero weight and no defined strain, here as there
    bad_r = ~np.isfinite(eps_r).all(axis=1)
    bad = ~np.isfinite(pts[:, :6]).all(axis=1)
    np.testing.assert_array_equal(bad, bad_r)
    assert (jw_r[bad_r] == 0.0).all() and (pts[bad, 6] == 0.0).all()
    ok = ~bad_r
    for got, ref in ((pts[ok, :3], eps_r[ok]), (pts[ok, 3:6], sig_r[ok])):
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    # homogenised response: J W-weighted averages over the live points
    w = jw_r[ok]
    for k, ref in enumerate((eps_r[ok], sig_r[ok])):
        avg = (w[:, None] * ref).sum(axis=0) / w.sum()
        np.testing.assert_allclose(mean[3 * k:3 * k + 3], avg, rtol=1e-12, atol=1e-12 * np.abs(avg).max())
    np.testing.assert_allclose(mean[6], w.sum(), rtol=1e-13)
    ctx.close()


def test_golden_with_collapsed_children_is_covered():
    g = golden("linear_3inc.npz")
    assert (~np.isfinite(g["qp.strain"])).any() and (g["qp.jw"] == 0.0).any()


def test_recovery_is_bit_reproducible():
    _, ctx = _with_reference_solution("linear_3inc.npz")
    a = ctx.compute_stress_strain()
    b = ctx.compute_stress_strain()
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])
    ctx.close()


def test_average_strain_equals_applied_strain_at_full_size():
    # 512 x 512 grid with 100 inclusions, solved on the device: the average
    # strain xx is the boundary integral of u_x n_x, the applied strain, for
    # any continuous field, converged or not; the area is the RVE's
    rve = config1()
    prob = pb.ProblemLinearElasticity(rve)
    prob.init()
    prob.get_solver().configure(rtol=1e-10)
    prob.solve_problem()
    pts, off, mean = prob.compute_stress_strain()
    area = (rve.x1 - rve.x0) * (rve.y1 - rve.y0)
    assert abs(mean[6] - area) <= 1e-12 * area
    assert abs(mean[0] - rve.strain) <= 1e-10 * rve.strain
    assert pts.shape[0] == off[-1] and np.isfinite(pts[:, 6]).all()
    prob.ctx.close()
