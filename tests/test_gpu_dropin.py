"""The reference's own Problem -- its mesh generation, IGFEM preprocessing,
DofObject numbering, boundary conditions and output NodalData -- with this
library's solver below it (oracle/integration/solver_gpu.h, linked into the
reference's driver by `make -f oracle/Makefile.ref dropin`): the K blocks the
library scatters into the reference's PETSc matrices, the solution and the
reactions the reference then holds, against the reference's own CPU run of
the same input (golden fixtures).  The binding also checks, node by node,
that the library's DOF map is the reference DofObject's.

Tolerances as for the library's own parity: K relative Frobenius 1e-12, U
relative 1e-8 (device solve to 1e-12), reactions 1e-8 relative."""
import os

import numpy as np
import pytest

import refio
from helpers import golden, ref_full_K, rel_fro

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["linear_8x8.npz", "linear_3inc.npz", "linear_cfg0.npz"])
def test_reference_problem_with_the_device_solver(name):
    if not os.path.exists(refio.DROPIN_DRIVER):
        pytest.skip("drop-in driver not built (make -f oracle/Makefile.ref dropin, needs the reference sources)")
    g = golden(name)
    nx = int(g["cfg.nx"][0])
    incs = [tuple(float(v) for v in row) for row in g["cfg.inc"]]
    r = refio.run(dict(nx=nx, ny=nx, E_matrix=3000.0, nu_matrix=0.35, strain=0.01, problem="linear", inclusions=incs),
                  driver=refio.DROPIN_DRIVER)
    assert r["gpu.rel_residual"][0] <= 1e-12
    # the reference's own mesh and numbering came out the same
    np.testing.assert_array_equal(r["dof.node"], g["dof.node"])
    np.testing.assert_array_equal(r["dof.enr"], g["dof.enr"])
    assert rel_fro(ref_full_K(r), ref_full_K(g)) <= 1e-12
    u = np.concatenate([r["U.f"], r["U.p"]])
    uref = np.concatenate([g["U.f"], g["U.p"]])
    assert np.linalg.norm(u - uref) / np.linalg.norm(uref) <= 1e-8
    np.testing.assert_allclose(r["F.p"], g["F.p"], rtol=0, atol=1e-8 * np.abs(g["F.p"]).max())
