"""Python mirror of the reference's Problem / Assembler / Solver call surface
for the IGFEM assembly and solve path, over the C ABI.

Reference surface (PIGFEM 4.6.1):
  Problem::init()                      src/Problem.cpp:105-316
  Problem::solve_problem()             src/Problem.cpp:400-418
  Problem::get_solver/get_assembler    include/Problem.h:149-153
  Assembler::assemble_linear(K)        src/Assembler.cpp:48-89
  Assembler::assemble_nonlinear(...)   src/Assembler.cpp:208-303
  Assembler::assemble_new_load_step    src/Assembler.cpp:554-663
  Solver::set_dparameter/iparameter    src/Solver.cpp:228-275
  PETScLinearKSPSolver::solve          src/SolverLinear.cpp:91-162
  SolverNonlinear::solve               src/SolverNonlinear.cpp:111-397

Errors follow the reference's convention of status codes turned into
exceptions (PgError) instead of err_message + exit.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr, u8ptr, lib
from .rve import RVE


class Mesh:
    """IGFEM mesh: Mesh::generate_mesh + the IGFEM steps of Problem::init
    (node/element detection, enrichment) + DOF numbering and sparsity
    (Problem::setup).  Built on the host (pg_mesh_build) or, with
    device=<GPU index>, on that GPU (pg_mesh_build_device): the same mesh bit
    for bit."""

    def __init__(self, rve: RVE, device: Optional[int] = None):
        self.rve = rve
        self._keep = []
        inc = rve.inclusions
        cx = np.ascontiguousarray([c[0] for c in inc], dtype=np.float64)
        cy = np.ascontiguousarray([c[1] for c in inc], dtype=np.float64)
        rr = np.ascontiguousarray([c[2] for c in inc], dtype=np.float64)
        im = np.ascontiguousarray([c[3] for c in inc], dtype=np.int32)
        E = np.ascontiguousarray([m[0] for m in rve.materials], dtype=np.float64)
        nu = np.ascontiguousarray([m[1] for m in rve.materials], dtype=np.float64)
        d = _lib.RveDesc()
        d.nx, d.ny = rve.nx, rve.ny
        d.x0, d.x1, d.y0, d.y1 = rve.x0, rve.x1, rve.y0, rve.y1
        d.n_inclusions = len(inc)
        d.inc_cx, d.inc_cy, d.inc_r, d.inc_mat = dptr(cx), dptr(cy), dptr(rr), iptr(im)
        d.n_materials = len(rve.materials)
        d.mat_E, d.mat_nu = dptr(E), dptr(nu)
        d.matrix_mat = rve.matrix_mat
        d.plane_strain = 1 if rve.plane_strain else 0
        d.cohesive = 1 if rve.cohesive else 0
        d.coh_law = rve.coh_law
        for k, v in enumerate(rve.coh_params[:5]):
            d.coh_params[k] = v
        d.strain = rve.strain
        h = C.c_void_p()
        if device is None:
            check(lib.pg_mesh_build(C.byref(d), C.byref(h)), "pg_mesh_build")
        else:
            check(lib.pg_mesh_build_device(C.byref(d), int(device), C.byref(h)), "pg_mesh_build_device")
        self.handle = h
        info = _lib.MeshInfo()
        check(lib.pg_mesh_info_get(h, C.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in _lib.MeshInfo._fields_}

    # held by the class, so that a mesh collected while the interpreter shuts
    # down (module globals already cleared) is still released
    _destroy = lib.pg_mesh_destroy

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._destroy(h)
            self.handle = None

    def export(self) -> Dict[str, np.ndarray]:
        i = self.info
        nn, ne, nd, nc, nb = i["n_nodes"], i["n_elements"], i["n_dof"], i["n_cut_elements"], i["n_blocks"]
        xy = np.zeros(2 * nn)
        conn = np.zeros(3 * ne, np.int32)
        emat = np.zeros(ne, np.int32)
        ecut = np.zeros(ne, np.int32)
        ref = np.zeros(nd, np.int32)
        fixed = np.zeros(nd, np.uint8)
        ubar = np.zeros(nd)
        check(lib.pg_mesh_export(self.handle, dptr(xy), iptr(conn), iptr(emat), iptr(ecut), iptr(ref),
                                 u8ptr(fixed), dptr(ubar)))
        ce = np.zeros(max(nc, 1), np.int32)
        ct = np.zeros(max(nc, 1), np.int32)
        cenr = np.zeros(max(nc, 1) * 12, np.int32)
        cmat = np.zeros(max(nc, 1) * 4, np.int32)
        cq0 = np.zeros(max(nc, 1), np.int32)
        check(lib.pg_mesh_export_cut(self.handle, iptr(ce), iptr(ct), iptr(cenr), iptr(cmat), iptr(cq0)))
        rp = np.zeros(nn + 1, np.int32)
        col = np.zeros(max(nb, 1), np.int32)
        check(lib.pg_mesh_export_pattern(self.handle, iptr(rp), iptr(col)))
        return dict(xy=xy.reshape(-1, 2), conn=conn.reshape(-1, 3), elem_mat=emat, elem_cut=ecut, ref_dof=ref,
                    fixed=fixed.astype(bool), ubar=ubar, cut_elem=ce[:nc], cut_tmpl=ct[:nc],
                    cut_enr=cenr[:12 * nc].reshape(-1, 12), cut_child_mat=cmat[:4 * nc].reshape(-1, 4),
                    cut_coh_qp0=cq0[:nc], row_ptr=rp, col=col[:nb],
                    n_regular_nodes=i["n_regular_nodes"], n_free=i["n_free_dof"])


def template_table() -> np.ndarray:
    n = C.c_int32()
    check(lib.pg_template_table(None, C.byref(n)))
    out = np.zeros(80 * n.value, np.int32)
    check(lib.pg_template_table(iptr(out), C.byref(n)))
    return out.reshape(n.value, 80)


class DeviceContext:
    """Device state of one mesh (Solver::setup on the GPU)."""

    def __init__(self, mesh: Mesh, device: int = 0):
        self.mesh = mesh
        h = C.c_void_p()
        check(lib.pg_ctx_create(mesh.handle, device, C.byref(h)), "pg_ctx_create")
        self.handle = h
        self.info = mesh.info

    _destroy = lib.pg_ctx_destroy  # (as Mesh._destroy)

    def close(self):
        if getattr(self, "handle", None):
            self._destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def sync(self):
        check(lib.pg_ctx_sync(self.handle))

    def matrix_values(self) -> np.ndarray:
        v = np.zeros(4 * self.info["n_blocks"])
        check(lib.pg_get_matrix(self.handle, dptr(v)))
        return v

    def vector(self, which: int = 0) -> np.ndarray:
        v = np.zeros(self.info["n_dof"])
        check(lib.pg_get_vector(self.handle, which, dptr(v)))
        return v

    def set_vector(self, which: int, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float64)
        check(lib.pg_set_vector(self.handle, which, dptr(v)))

    def isv(self, committed: bool = True) -> np.ndarray:
        v = np.zeros(max(1, self.info["n_cohesive_qp"]))
        check(lib.pg_get_isv(self.handle, 1 if committed else 0, dptr(v)))
        return v[: self.info["n_cohesive_qp"]]


def _stress_strain(ctx, U_dev: Optional[int] = None, points: bool = True):
    """Problem::compute_stress_strain (src/Problem.cpp:428-534) over every
    element at once, and the homogenised response.  Returns (points, offsets,
    mean): points[n, 7] = strain xx, yy, xy (engineering), stress xx, yy, xy,
    J W per volumetric quadrature point in the reference's order (NaN strain
    and stress at zero-weight points of collapsed children); offsets[e] the
    first point of element e; mean[7] = the J W-weighted averages of strain
    and stress and the total J W."""
    n = C.c_int64()
    off = np.zeros(ctx.info["n_elements"] + 1, np.int32)
    check(lib.pg_stress_strain(ctx.handle, None, None, C.byref(n), iptr(off), None), "pg_stress_strain")
    pts = np.zeros((n.value, 7)) if points else None
    mean = np.zeros(7)
    ptr = C.cast(C.c_void_p(U_dev), _lib._dp) if U_dev else None
    check(lib.pg_stress_strain(ctx.handle, ptr, dptr(pts) if points else None, None, None, dptr(mean)),
          "pg_stress_strain")
    return pts, off, mean


DeviceContext.compute_stress_strain = _stress_strain


def _set_isv(ctx, v, committed=True):
    v = np.ascontiguousarray(v, dtype=np.float64)
    check(lib.pg_set_isv(ctx.handle, 1 if committed else 0, dptr(v)))


DeviceContext.set_isv = _set_isv


class Assembler:
    """Assembler surface (include/Assembler.h:41-51)."""

    def __init__(self, ctx: DeviceContext):
        self.ctx = ctx

    def assemble_linear(self, stream: Optional[int] = None) -> None:
        check(lib.pg_assemble_linear(self.ctx.handle, stream), "assemble_linear")

    def assemble_nonlinear(self, dt: float, assemble_func: bool = True, assemble_jac: bool = True,
                           U_dev: Optional[int] = None) -> None:
        ptr = C.cast(C.c_void_p(U_dev), _lib._dp) if U_dev else None
        check(lib.pg_assemble_nonlinear(self.ctx.handle, ptr, dt, int(assemble_func), int(assemble_jac), None),
              "assemble_nonlinear")

    def assemble_new_load_step(self, current_time_frac: float) -> None:
        check(lib.pg_new_load_step(self.ctx.handle, current_time_frac), "assemble_new_load_step")


class Solver:
    """Solver surface with the reference's parameter names
    (Solver::set_dparameter / set_iparameter, src/Solver.cpp:228-275)."""

    def __init__(self, ctx: DeviceContext):
        self.ctx = ctx
        self.cfg = _lib.SolverCfg()
        lib.pg_solver_cfg_default(C.byref(self.cfg))
        self.dparams = {"rel_tol": 1e-8, "abs_tol": 1e-8, "T_final": 1.0, "max_time_step": 1.0,
                        "min_time_step": 1e-6}
        self.iparams = {"max_iter": 40}
        self.stats = _lib.SolveStats()

    def set_dparameter(self, name: str, val: float) -> None:
        self.dparams[name] = float(val)

    def set_iparameter(self, name: str, val: int) -> None:
        self.iparams[name] = int(val)

    def configure(self, precision: int = _lib.PG_PRECISION_FP64, precond: int = _lib.PG_PREC_BLOCK_JACOBI,
                  rtol: float = 1e-8, inner_rtol: float = 1e-4, max_iter: int = 200000,
                  check_every: int = 64, deterministic: bool = True) -> None:
        self.cfg.precision = precision
        self.cfg.precond = precond
        self.cfg.rtol = rtol
        self.cfg.inner_rtol = inner_rtol
        self.cfg.max_iter = max_iter
        self.cfg.check_every = check_every
        self.cfg.deterministic = int(deterministic)

    def solve_linear(self) -> _lib.SolveStats:
        check(lib.pg_solve_linear(self.ctx.handle, C.byref(self.cfg), C.byref(self.stats)), "pg_solve_linear")
        return self.stats


class ProblemLinearElasticity:
    """Problem::init / solve_problem for the linear elastic IGFEM RVE."""

    def __init__(self, rve: RVE, device: int = 0):
        self.rve = rve
        self.device = device
        self.mesh: Optional[Mesh] = None
        self.ctx: Optional[DeviceContext] = None

    def init(self) -> None:
        self.mesh = Mesh(self.rve)
        self.ctx = DeviceContext(self.mesh, self.device)
        self.assembler = Assembler(self.ctx)
        self.solver = Solver(self.ctx)

    def get_solver(self) -> Solver:
        return self.solver

    def get_assembler(self) -> Assembler:
        return self.assembler

    def solve_problem(self) -> _lib.SolveStats:
        self.assembler.assemble_linear()
        return self.solver.solve_linear()

    def get_solution(self) -> np.ndarray:
        return self.ctx.vector(0)

    def compute_stress_strain(self, points: bool = True):
        """Strain and stress at every volumetric quadrature point of the
        current solution, and their volume averages (see
        DeviceContext.compute_stress_strain)."""
        return self.ctx.compute_stress_strain(points=points)


class ProblemNonlinearStructural:
    """Problem::init / solve_problem for cohesive RVEs: load stepping with
    Newton (SolverNonlinear::solve, src/SolverNonlinear.cpp:111-397)."""

    def __init__(self, rve: RVE, device: int = 0):
        self.rve = rve
        self.device = device
        self.mesh: Optional[Mesh] = None
        self.ctx: Optional[DeviceContext] = None
        self.cfg = _lib.NewtonCfg()
        lib.pg_newton_cfg_default(C.byref(self.cfg))

    def init(self) -> None:
        self.mesh = Mesh(self.rve)
        self.ctx = DeviceContext(self.mesh, self.device)
        self.assembler = Assembler(self.ctx)
        self.solver = Solver(self.ctx)

    def get_solver(self) -> Solver:
        return self.solver

    def get_assembler(self) -> Assembler:
        return self.assembler

    def configure(self, **kw) -> None:
        for k, v in kw.items():
            if not hasattr(self.cfg, k):
                raise KeyError(k)
            setattr(self.cfg, k, v)

    def solve_problem(self, max_records: int = 4096):
        recs = (_lib.StepStats * max_records)()
        n = C.c_int32()
        check(lib.pg_solve_nonlinear(self.ctx.handle, C.byref(self.cfg), recs, max_records, C.byref(n)),
              "pg_solve_nonlinear")
        return [recs[i] for i in range(min(n.value, max_records))]

    def load_step(self, t_frac: float, dt: float) -> _lib.StepStats:
        st = _lib.StepStats()
        check(lib.pg_newton_load_step(self.ctx.handle, t_frac, dt, C.byref(self.cfg), C.byref(st)),
              "pg_newton_load_step")
        return st

    def commit(self) -> None:
        check(lib.pg_commit_isv(self.ctx.handle))

    def get_solution(self) -> np.ndarray:
        return self.ctx.vector(0)

    def compute_stress_strain(self, points: bool = True):
        """Strain and stress at every volumetric quadrature point of the
        current solution, and their volume averages (see
        DeviceContext.compute_stress_strain)."""
        return self.ctx.compute_stress_strain(points=points)


class Writer_ASCII_VTK:
    """Writer_ASCII_VTK (src/Writer_ASCII_VTK.cpp, src/Writer_VTK.cpp): the
    legacy ASCII VTK file of a problem's current state, in the reference's
    layout and number format."""

    def __init__(self, prob):
        self.prob = prob

    def store_mesh(self) -> None:
        """The mesh is fixed once the context exists: nothing to store."""

    def write(self, filename: str, curr_t: float) -> None:
        check(lib.pg_write_vtk(self.prob.ctx.handle, filename.encode(), float(curr_t)), "pg_write_vtk")


class WriterCohesiveOpenings:
    """WriterCohesiveOpenings (src/WriterCohesiveOpenings.cpp): per cohesive
    sub-element its inclusion, angle and normalised midpoint opening, as CSV."""

    def __init__(self, prob):
        self.prob = prob

    def store_mesh(self) -> None:
        """The mesh is fixed once the context exists: nothing to store."""

    def write(self, filename: str, curr_t: float = 0.0) -> None:
        check(lib.pg_write_cohesive_openings(self.prob.ctx.handle, filename.encode()), "pg_write_cohesive_openings")
