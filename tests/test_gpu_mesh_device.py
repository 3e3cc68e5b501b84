"""IGFEM preprocessing and sparsity on the GPU (pg_mesh_build_device) against
the host builder (pg_mesh_build), which is itself pinned node for node to
the reference's enriched mesh (tests/test_host_mesh.py): every exported
array -- coordinates, connectivity, materials, cut templates, enrichment
slots, DOF numbering, Dirichlet data, block pattern -- must be equal bit for
bit, and the contexts made from the two meshes must assemble identical K."""
import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from helpers import golden, rve_from_golden
from pigfem_assignment_b200.rve import RVE, config0, config1, config2, config3_rves, config4

pytestmark = pytest.mark.gpu


def _cases():
    yield "config0 (moved nodes)", config0()
    yield "config1", config1()
    yield "config2 cohesive", config2()
    yield "golden 3 inclusions (node on an interface)", rve_from_golden(golden("linear_3inc.npz"))
    yield "golden cohesive 16x16", rve_from_golden(golden("cohesive_16x16.npz"), cohesive=True)
    yield "two close inclusions", RVE(nx=40, ny=40, inclusions=[(0.3, 0.5, 0.2, 1), (0.72, 0.5, 0.2, 1)], strain=0.01)
    yield "thin strip", RVE(nx=33, ny=2, inclusions=[(0.5, 0.5, 0.3, 1)], strain=0.01)
    for k, r in enumerate(config3_rves(3, 6)):
        yield f"config3 rve {k}", r
    yield "config4 geometry", config4()


CASES = list(_cases())


@pytest.mark.parametrize("name,rve", CASES, ids=[c[0] for c in CASES])
def test_device_mesh_equals_host_mesh(name, rve):
    mh = pb.Mesh(rve)
    md = pb.Mesh(rve, device=0)
    assert md.info == mh.info, name
    eh, ed = mh.export(), md.export()
    assert eh.keys() == ed.keys()
    for k in eh:
        a, b = np.asarray(eh[k]), np.asarray(ed[k])
        assert a.shape == b.shape, (name, k)
        assert np.array_equal(a, b), (name, k)


@pytest.mark.parametrize("name,rve", [CASES[0], CASES[4], CASES[5]], ids=[CASES[i][0] for i in (0, 4, 5)])
def test_contexts_of_both_meshes_assemble_the_same_bits(name, rve):
    Ks = []
    for dev in (None, 0):
        m = pb.Mesh(rve, device=dev)
        ctx = pb.DeviceContext(m)
        if rve.cohesive:
            rng = np.random.default_rng(2)
            ctx.set_vector(0, 1e-4 * rng.standard_normal(m.info["n_dof"]))
            pb.Assembler(ctx).assemble_nonlinear(0.1, True, True)
            Ks.append((ctx.matrix_values(), ctx.vector(1)))
        else:
            pb.Assembler(ctx).assemble_linear()
            Ks.append((ctx.matrix_values(), None))
        ctx.close()
    assert np.array_equal(Ks[0][0], Ks[1][0]), name
    if Ks[0][1] is not None:
        assert np.array_equal(Ks[0][1], Ks[1][1]), name
