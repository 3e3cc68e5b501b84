// The binding a maintainer would add to PIGFEM 4.6.1 to run its linear
// elastic IGFEM path on the B200 library (include/pigfem_b200.h), compiled
// here against the reference's own headers (PIGFEM4.6.1/include) and linked
// with its unmodified objects (oracle/Makefile.ref) -- test infrastructure
// that shows the C ABI is a drop-in below the reference's Problem.
//
// The reference's Assembler::assemble_linear is not virtual, so the seam is
// the solver: Problem::init builds its solver through the virtual
// Problem::generate_solver (include/Problem.h:270), and
// ProblemLinearElasticityGPU returns SolverGPULinear there.  Everything above
// the solver -- Mesh, the IGFEM preprocessing, DofObject, BoundaryObject,
// Problem::init / setup / solve_problem, the output NodalData -- stays the
// reference's.  SolverGPULinear::solve replaces PETScLinearKSPSolver::solve
// (src/SolverLinear.cpp:91-162): the library assembles K and solves on the
// device; the K blocks, the solution and the reactions are then scattered into
// the reference's PETSc objects (_K.ff/fp/pf/pp, _U.f/p, _F_ext.p) by the
// reference's own DOF numbers, and stored into the Problem's NodalData with
// Solver::store_solution, so every later reader of the reference sees the
// state its own solve would have left.
#pragma once

#include <vector>

#include "ProblemLinearElasticity.h"
#include "SolverLinear.h"
#include "pigfem_b200.h"

class SolverGPULinear : public PETScLinearKSPSolver {
  public:
    // desc: the RVE the reference's mesh was generated from (structured grid,
    // circles, materials, applied strain); rtol: the device solve's target
    SolverGPULinear(const pg_rve_desc& desc, int device, double rtol);
    virtual ~SolverGPULinear();
    virtual PetscErrorCode solve();

    const pg_solve_stats& stats() const { return _stats; }
    // the reference's Problem::solve_problem drops the solver's status: the
    // last solve's is kept here
    PetscErrorCode status() const { return _status; }

  private:
    // the library's mesh and device context, and the check that its DOF map
    // is the reference DofObject's (DofObject::get_global_dof)
    PetscErrorCode ensure_context();
    // pg_get_matrix -> MatSetValues into _K.ff/fp/pf/pp
    PetscErrorCode scatter_to_petsc();
    // a library-ordered vector -> the reference's free / prescribed Vecs
    PetscErrorCode scatter_vec(const std::vector<double>& v, Vec& f, Vec& p, bool free_part);
    // the Problem's NodalData solution -> the device (library order)
    PetscErrorCode upload_solution(NodalData* sol);

    pg_rve_desc _desc;
    std::vector<double> _inc_cx, _inc_cy, _inc_r, _mat_E, _mat_nu;
    std::vector<int32_t> _inc_mat;
    int _device;
    double _rtol;
    pg_mesh* _mesh = nullptr;
    pg_ctx* _ctx = nullptr;
    pg_mesh_info _info{};
    std::vector<int32_t> _ref_dof, _row_ptr, _col;
    pg_solve_stats _stats{};
    PetscErrorCode _status = 0;
    PetscErrorCode solve_on_device();
};

class ProblemLinearElasticityGPU : public ProblemLinearElasticity {
  public:
    ProblemLinearElasticityGPU(const pg_rve_desc& desc, int device, double rtol)
        : _desc(desc), _device(device), _rtol(rtol) {}

  protected:
    // ProblemLinear::generate_solver (src/ProblemLinear.cpp:31-34) builds a
    // PETScLinearKSPSolver; this builds the device solver instead
    virtual void generate_solver();

  private:
    pg_rve_desc _desc;
    int _device;
    double _rtol;
};
