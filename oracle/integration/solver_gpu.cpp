// SolverGPULinear / ProblemLinearElasticityGPU: see solver_gpu.h.
#include "solver_gpu.h"

#include <cstdio>
#include <string>

#include "DofObject.h"
#include "Mesh.h"
#include "NodalData.h"
#include "Problem.h"

namespace {

PetscErrorCode pg_fail(int rc, const char* what) {
    fprintf(stderr, "SolverGPULinear: %s failed (status %d): %s\n", what, rc, pg_last_error());
    return (PetscErrorCode)(1000 + rc);
}

}  // namespace

SolverGPULinear::SolverGPULinear(const pg_rve_desc& desc, int device, double rtol)
    : _desc(desc), _device(device), _rtol(rtol) {
    // own copies of the description's arrays
    const int ni = desc.n_inclusions, nm = desc.n_materials;
    _inc_cx.assign(desc.inc_cx, desc.inc_cx + ni);
    _inc_cy.assign(desc.inc_cy, desc.inc_cy + ni);
    _inc_r.assign(desc.inc_r, desc.inc_r + ni);
    _inc_mat.assign(desc.inc_mat, desc.inc_mat + ni);
    _mat_E.assign(desc.mat_E, desc.mat_E + nm);
    _mat_nu.assign(desc.mat_nu, desc.mat_nu + nm);
    _desc.inc_cx = _inc_cx.data();
    _desc.inc_cy = _inc_cy.data();
    _desc.inc_r = _inc_r.data();
    _desc.inc_mat = _inc_mat.data();
    _desc.mat_E = _mat_E.data();
    _desc.mat_nu = _mat_nu.data();
}

SolverGPULinear::~SolverGPULinear() {
    if (_ctx) pg_ctx_destroy(_ctx);
    if (_mesh) pg_mesh_destroy(_mesh);
}

PetscErrorCode SolverGPULinear::ensure_context() {
    if (_ctx) return 0;
    int rc = pg_mesh_build(&_desc, &_mesh);
    if (rc) return pg_fail(rc, "pg_mesh_build");
    pg_mesh_info_get(_mesh, &_info);
    _ref_dof.resize(_info.n_dof);
    rc = pg_mesh_export(_mesh, nullptr, nullptr, nullptr, nullptr, _ref_dof.data(), nullptr, nullptr);
    if (rc) return pg_fail(rc, "pg_mesh_export");
    _row_ptr.resize(_info.n_nodes + 1);
    _col.resize(_info.n_blocks);
    rc = pg_mesh_export_pattern(_mesh, _row_ptr.data(), _col.data());
    if (rc) return pg_fail(rc, "pg_mesh_export_pattern");
    // the library's DOF map must be the reference DofObject's, node for node
    Mesh* mesh = _prob->get_mesh();
    DofObject* dofs = _prob->get_dofs();
    if ((id_type)_info.n_regular_nodes != mesh->n_global_nodes() ||
        (id_type)_info.n_enrichment_nodes != mesh->n_global_enrich_nodes() ||
        (id_type)_info.n_free_dof != dofs->n_global_free_dofs()) {
        fprintf(stderr, "SolverGPULinear: the library's mesh differs from the reference's\n");
        return 1;
    }
    for (int n = 0; n < _info.n_nodes; ++n) {
        const id_type id = n < _info.n_regular_nodes ? (id_type)n : ENRICH_START + (id_type)(n - _info.n_regular_nodes);
        for (int d = 0; d < 2; ++d)
            if ((id_type)_ref_dof[2 * n + d] != dofs->get_global_dof(id, d)) {
                fprintf(stderr, "SolverGPULinear: DOF %d of node %d: library %d, reference %lu\n", d, n,
                        _ref_dof[2 * n + d], (unsigned long)dofs->get_global_dof(id, d));
                return 1;
            }
    }
    rc = pg_ctx_create(_mesh, _device, &_ctx);
    if (rc) return pg_fail(rc, "pg_ctx_create");
    return 0;
}

PetscErrorCode SolverGPULinear::scatter_to_petsc() {
    std::vector<double> vals(4 * (size_t)_info.n_blocks);
    int rc = pg_get_matrix(_ctx, vals.data());
    if (rc) return pg_fail(rc, "pg_get_matrix");
    PetscErrorCode ierr;
    for (Mat* m : {&_K.ff, &_K.fp, &_K.pf, &_K.pp}) {
        ierr = MatZeroEntries(*m);CHKERRQ(ierr);
    }
    const PetscInt nf = (PetscInt)_info.n_free_dof;
    for (int a = 0; a < _info.n_nodes; ++a)
        for (int k = _row_ptr[a]; k < _row_ptr[a + 1]; ++k) {
            const int b = _col[k];
            for (int da = 0; da < 2; ++da)
                for (int db = 0; db < 2; ++db) {
                    const double v = vals[4 * (size_t)k + 2 * da + db];
                    if (v == 0.0) continue;
                    const PetscInt i = _ref_dof[2 * a + da], j = _ref_dof[2 * b + db];
                    Mat& M = i < nf ? (j < nf ? _K.ff : _K.fp) : (j < nf ? _K.pf : _K.pp);
                    ierr = MatSetValue(M, i < nf ? i : i - nf, j < nf ? j : j - nf, v, INSERT_VALUES);CHKERRQ(ierr);
                }
        }
    for (Mat* m : {&_K.ff, &_K.fp, &_K.pf, &_K.pp}) {
        ierr = MatAssemblyBegin(*m, MAT_FINAL_ASSEMBLY);CHKERRQ(ierr);
        ierr = MatAssemblyEnd(*m, MAT_FINAL_ASSEMBLY);CHKERRQ(ierr);
    }
    return 0;
}

PetscErrorCode SolverGPULinear::scatter_vec(const std::vector<double>& v, Vec& f, Vec& p, bool free_part) {
    PetscErrorCode ierr;
    const PetscInt nf = (PetscInt)_info.n_free_dof;
    for (int i = 0; i < _info.n_dof; ++i) {
        const PetscInt r = _ref_dof[i];
        if (r < nf && free_part) {
            ierr = VecSetValue(f, r, v[i], INSERT_VALUES);CHKERRQ(ierr);
        } else if (r >= nf) {
            ierr = VecSetValue(p, r - nf, v[i], INSERT_VALUES);CHKERRQ(ierr);
        }
    }
    ierr = VecAssemblyBegin(f);CHKERRQ(ierr);
    ierr = VecAssemblyEnd(f);CHKERRQ(ierr);
    ierr = VecAssemblyBegin(p);CHKERRQ(ierr);
    ierr = VecAssemblyEnd(p);CHKERRQ(ierr);
    return 0;
}

PetscErrorCode SolverGPULinear::upload_solution(NodalData* sol) {
    Mesh* mesh = _prob->get_mesh();
    std::vector<double> U(_info.n_dof, 0.0);
    for (int n = 0; n < _info.n_nodes; ++n) {
        const id_type id = n < _info.n_regular_nodes ? (id_type)n : ENRICH_START + (id_type)(n - _info.n_regular_nodes);
        const id_type l = mesh->global_to_local_node(id);
        for (int d = 0; d < 2; ++d) U[2 * n + d] = sol->get_value_local(l, d);
    }
    const int rc = pg_set_vector(_ctx, 0, U.data());
    return rc ? pg_fail(rc, "pg_set_vector") : 0;
}

// PETScLinearKSPSolver::solve (src/SolverLinear.cpp:91-162) on the device
PetscErrorCode SolverGPULinear::solve() {
    _status = solve_on_device();
    return _status;
}

PetscErrorCode SolverGPULinear::solve_on_device() {
    PetscErrorCode ierr = ensure_context();
    if (ierr) return ierr;
    // the Problem's current solution is the initial guess of the free DOFs
    ierr = upload_solution(_prob->get_solution());
    if (ierr) return ierr;
    int rc = pg_assemble_linear(_ctx, nullptr);
    if (rc) return pg_fail(rc, "pg_assemble_linear");
    pg_solver_cfg cfg;
    pg_solver_cfg_default(&cfg);
    cfg.precond = PG_PREC_MG;
    cfg.rtol = _rtol;
    rc = pg_solve_linear(_ctx, &cfg, &_stats);
    if (rc) return pg_fail(rc, "pg_solve_linear");
    // K into the reference's blocks, U into U.f / U.p (U.p: the prescribed values)
    ierr = scatter_to_petsc();
    if (ierr) return ierr;
    std::vector<double> U(_info.n_dof);
    rc = pg_get_vector(_ctx, 0, U.data());
    if (rc) return pg_fail(rc, "pg_get_vector");
    ierr = scatter_vec(U, _U.f, _U.p, true);
    if (ierr) return ierr;
    // reactions as the reference forms them: F_p = K_pf U_f + K_pp U_p
    Vec temp;
    ierr = VecDuplicate(_F_ext.p, &temp);CHKERRQ(ierr);
    ierr = MatMult(_K.pf, _U.f, temp);CHKERRQ(ierr);
    ierr = MatMult(_K.pp, _U.p, _F_ext.p);CHKERRQ(ierr);
    ierr = VecAXPY(_F_ext.p, 1.0, temp);CHKERRQ(ierr);
    ierr = VecDestroy(&temp);CHKERRQ(ierr);
    ierr = store_solution(_U, _prob->get_solution());CHKERRQ(ierr);
    ierr = store_solution(_F_ext, _prob->get_external_load());CHKERRQ(ierr);
    return 0;
}

void ProblemLinearElasticityGPU::generate_solver() {
    if (_solver != NULL) delete _solver;
    _solver = new SolverGPULinear(_desc, _device, _rtol);
}
