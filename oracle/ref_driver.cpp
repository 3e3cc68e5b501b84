// Oracle driver: runs the REFERENCE (PIGFEM 4.6.1, compiled unmodified from
// its own sources against the single-rank shim in oracle/ref_shim) through
// its own public API -- Mesh::generate_mesh, Mesh::add_inclusion,
// Problem::init, Problem::solve_problem -- the way PIGFEM4.6.1/Tests/Main.cpp
// does (materials :310-429, boundary conditions :433-450), and dumps what the
// reference computed: the enriched mesh, the DOF numbering, the assembled
// stiffness blocks K_ff/K_fp/K_pf/K_pp, load vectors, the solution, the
// cohesive internal state and per-phase timings.
//
// Test infrastructure only.  Output: a flat record file read by
// oracle/refio.py (name, dtype, count, raw data).
//
// Usage: pigfem_ref_driver <config.txt> <out.bin> <scratch_dir>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>
#include <algorithm>
#include <chrono>
#include <functional>
#include <deque>
#include <list>
#include <memory>
#include <new>

// The driver reads solver/mesh internals that the reference keeps private
// (e.g. Solver::_K).  This only changes access checking inside this
// translation unit; the reference objects themselves are built unmodified.
#define private public
#define protected public
#include "Mesh.h"
#include "elem.h"
#include "node.h"
#include "Problem.h"
#include "ProblemLinearElasticity.h"
#include "ProblemNonlinearStructural.h"
#include "BoundaryObject.h"
#include "DofObject.h"
#include "InclusionCircle.h"
#include "material_lei.h"
#include "Material_OPCohesive.h"
#include "Solver.h"
#include "SolverNonlinear.h"
#include "Assembler.h"
#include "InternalVars.h"
#include "Options.h"
#include "Utilities.h"
#include "SensitivityRightLoad.h"
#include "SensitivitySolver.h"
#include "SensitivityAdjoint.h"
#include "Writer_ASCII_VTK.h"
#include "WriterCohesiveOpenings.h"
#undef private
#undef protected
#ifdef PG_GPU_DROPIN
#include "integration/solver_gpu.h"
#endif

namespace {

struct Config {
    int nx = 8, ny = 8;
    double x0 = 0, x1 = 1, y0 = 0, y1 = 1;
    double E_m = 3000, nu_m = 0.35;
    int plane_strain = 1;
    double strain = 0.01;
    std::string problem = "linear";
    struct Inc { double cx, cy, r, E, nu; };
    std::vector<Inc> incs;
    double coh_sigma = 10, coh_delta = 1.5e-4, coh_beta = 1.0, coh_visc = 0.5;
    double T_final = 1.0, max_dt = 0.02, min_dt = 1e-6;
    int max_iter = 40;
    int assemble_repeats = 0;   // >0: time assemble_linear this many times (linear only)
    int dump_K = 1;
    double snes_rtol = 0.0, snes_stol = -1.0;  // > 0 / >= 0: the shim's SNES defaults (PETSc: 1e-8, 1e-8)
    std::string vtk_out, openings_out;  // non-empty: write the reference's VTK file / cohesive openings CSV there
    struct SensParam { int inc; std::string name; };
    std::vector<SensParam> sens;        // shape parameters ("X", "Y", "R") of SensitivityRightLoad
};

Config read_config(const char* path) {
    Config c;
    std::ifstream in(path);
    if (!in.good()) { fprintf(stderr, "cannot read %s\n", path); exit(2); }
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string k;
        if (!(ss >> k) || k[0] == '#') continue;
        if (k == "nx") ss >> c.nx;
        else if (k == "ny") ss >> c.ny;
        else if (k == "x0") ss >> c.x0;
        else if (k == "x1") ss >> c.x1;
        else if (k == "y0") ss >> c.y0;
        else if (k == "y1") ss >> c.y1;
        else if (k == "E_matrix") ss >> c.E_m;
        else if (k == "nu_matrix") ss >> c.nu_m;
        else if (k == "plane_strain") ss >> c.plane_strain;
        else if (k == "strain") ss >> c.strain;
        else if (k == "problem") ss >> c.problem;
        else if (k == "inc") { Config::Inc i; ss >> i.cx >> i.cy >> i.r >> i.E >> i.nu; c.incs.push_back(i); }
        else if (k == "coh_sigma") ss >> c.coh_sigma;
        else if (k == "coh_delta") ss >> c.coh_delta;
        else if (k == "coh_beta") ss >> c.coh_beta;
        else if (k == "coh_visc") ss >> c.coh_visc;
        else if (k == "T_final") ss >> c.T_final;
        else if (k == "max_dt") ss >> c.max_dt;
        else if (k == "min_dt") ss >> c.min_dt;
        else if (k == "max_iter") ss >> c.max_iter;
        else if (k == "assemble_repeats") ss >> c.assemble_repeats;
        else if (k == "dump_K") ss >> c.dump_K;
        else if (k == "snes_rtol") ss >> c.snes_rtol;
        else if (k == "snes_stol") ss >> c.snes_stol;
        else if (k == "vtk_out") ss >> c.vtk_out;
        else if (k == "sens") { Config::SensParam p; ss >> p.inc >> p.name; c.sens.push_back(p); }
        else if (k == "openings_out") ss >> c.openings_out;
        else { fprintf(stderr, "unknown config key %s\n", k.c_str()); exit(2); }
    }
    return c;
}

struct Out {
    FILE* f;
    void rec(const std::string& name, char dt, const void* data, int64_t count) {
        int32_t nl = (int32_t)name.size();
        fwrite(&nl, 4, 1, f);
        fwrite(name.data(), 1, nl, f);
        fwrite(&dt, 1, 1, f);
        fwrite(&count, 8, 1, f);
        size_t es = dt == 'd' ? 8 : (dt == 'q' ? 8 : 4);
        if (count) fwrite(data, es, (size_t)count, f);
    }
    void d(const std::string& n, const std::vector<double>& v) { rec(n, 'd', v.data(), (int64_t)v.size()); }
    void i(const std::string& n, const std::vector<int32_t>& v) { rec(n, 'i', v.data(), (int64_t)v.size()); }
    void d1(const std::string& n, double v) { rec(n, 'd', &v, 1); }
    void i1(const std::string& n, int32_t v) { rec(n, 'i', &v, 1); }
};

void dump_mat(Out& o, const std::string& name, Mat A) {
    std::vector<int32_t> rp(1, 0), ci;
    std::vector<double> va;
    const int m = pgshim_mat_rows(A);
    for (int r = 0; r < m; ++r) {
        int k = pgshim_mat_row_nnz(A, r);
        std::vector<PetscInt> cs(k);
        std::vector<PetscScalar> vs(k);
        pgshim_mat_row(A, r, cs.data(), vs.data());
        for (int t = 0; t < k; ++t) { ci.push_back(cs[t]); va.push_back(vs[t]); }
        rp.push_back((int32_t)ci.size());
    }
    o.i(name + ".shape", {m, (int32_t)pgshim_mat_cols(A)});
    o.i(name + ".rowptr", rp);
    o.i(name + ".col", ci);
    o.d(name + ".val", va);
}

void dump_vec(Out& o, const std::string& name, Vec v) {
    const int n = pgshim_vec_size(v);
    const double* p = pgshim_vec_data(v);
    o.d(name, std::vector<double>(p, p + n));
}

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) { fprintf(stderr, "usage: %s config out.bin scratch_dir\n", argv[0]); return 2; }
    Config cfg = read_config(argv[1]);
    // SNES tolerances the shim takes as its defaults (see SNESCreate there)
    char tolbuf[64];
    if (cfg.snes_rtol > 0.0) {
        snprintf(tolbuf, sizeof tolbuf, "%.17g", cfg.snes_rtol);
        setenv("PGSHIM_SNES_RTOL", tolbuf, 1);
    }
    if (cfg.snes_stol >= 0.0) {
        snprintf(tolbuf, sizeof tolbuf, "%.17g", cfg.snes_stol);
        setenv("PGSHIM_SNES_STOL", tolbuf, 1);
    }
    std::string scratch = std::string(argv[3]);
    if (scratch.back() != '/') scratch += "/";

    int pargc = 9;
    std::string a0 = "pigfem_ref_driver", f1 = "-OUT_FOLDER", f2 = "-WRITE_VTK", v2 = "false",
                f3 = "-WRITE_TO_SCREEN", v3 = "false", f4 = "-LOG", v4 = "log.txt";
    char* pargv_arr[] = {&a0[0], &f1[0], &scratch[0], &f2[0], &v2[0], &f3[0], &v3[0], &f4[0], &v4[0], nullptr};
    char** pargv = pargv_arr;

    Mesh mesh(&pargc, &pargv);
    const bool cohesive = (cfg.problem == "cohesive");
    // Problem::Problem() (PIGFEM4.6.1/src/Problem.cpp:42-53) leaves
    // _internal_vars uninitialised and Problem::init() deletes it
    // (Problem.cpp:186); with an indeterminate pointer that crashes (the
    // reference's own recorded run, Test.error.txt:19-40, dies right there).
    // Constructing the object in zeroed storage makes the pointer NULL without
    // touching the reference's code.
    Problem* problem;
    if (cohesive) {
        void* mem = calloc(1, sizeof(ProblemNonlinearStructural));
        problem = new (mem) ProblemNonlinearStructural;
    } else {
#ifdef PG_GPU_DROPIN
        // the same Problem with the B200 library's solver below it
        // (oracle/integration/solver_gpu.h); the description is the one this
        // driver generates the reference's mesh from
        static std::vector<double> cx, cy, rr, mE, mnu;
        static std::vector<int32_t> im;
        std::map<std::pair<double, double>, int> mat_of;
        mE.push_back(cfg.E_m);
        mnu.push_back(cfg.nu_m);
        for (const auto& ic : cfg.incs) {
            auto key = std::make_pair(ic.E, ic.nu);
            if (!mat_of.count(key)) {
                mat_of[key] = (int)mE.size();
                mE.push_back(ic.E);
                mnu.push_back(ic.nu);
            }
            cx.push_back(ic.cx);
            cy.push_back(ic.cy);
            rr.push_back(ic.r);
            im.push_back(mat_of[key]);
        }
        pg_rve_desc desc{};
        desc.nx = cfg.nx;
        desc.ny = cfg.ny;
        desc.x0 = cfg.x0;
        desc.x1 = cfg.x1;
        desc.y0 = cfg.y0;
        desc.y1 = cfg.y1;
        desc.n_inclusions = (int32_t)cx.size();
        desc.inc_cx = cx.data();
        desc.inc_cy = cy.data();
        desc.inc_r = rr.data();
        desc.inc_mat = im.data();
        desc.n_materials = (int32_t)mE.size();
        desc.mat_E = mE.data();
        desc.mat_nu = mnu.data();
        desc.matrix_mat = 0;
        desc.plane_strain = cfg.plane_strain;
        desc.strain = cfg.strain;
        void* mem = calloc(1, sizeof(ProblemLinearElasticityGPU));
        problem = new (mem) ProblemLinearElasticityGPU(desc, 0, 1e-12);
#else
        void* mem = calloc(1, sizeof(ProblemLinearElasticity));
        problem = new (mem) ProblemLinearElasticity;
#endif
    }
    problem->set_parameter("plane_strain", cfg.plane_strain);
    problem->attach_mesh(&mesh);
    problem->getOptions()->parseInput(pargc, pargv);

    // Inclusions (PIGFEM4.6.1/Tests/Main.cpp read_csv/add_circle).  One
    // material per distinct (E, nu); inclusions sharing it share the material.
    std::vector<LinearElasticIsotropicMaterial*> inc_mats;
    std::map<std::pair<double, double>, std::string> mat_names;
    for (size_t k = 0; k < cfg.incs.size(); ++k) {
        const auto& ic = cfg.incs[k];
        auto key = std::make_pair(ic.E, ic.nu);
        auto* m = new LinearElasticIsotropicMaterial;
        m->set_parameter("E", ic.E);
        m->set_parameter("nu", ic.nu);
        std::string name;
        if (mat_names.count(key)) name = mat_names[key];
        else { name = "Carbon" + std::to_string(mat_names.size()); mat_names[key] = name; }
        m->set_name(name);
        inc_mats.push_back(m);
        Circle_Inclusion circle;
        circle.set_material(m);
        std::vector<double> center = {ic.cx, ic.cy};
        circle.set_vec_parameter("center", center);
        circle.set_parameter("r", ic.r);
        mesh.add_inclusion(&circle);
    }

    mesh.generate_mesh(TRI3, cfg.x0, cfg.x1, cfg.nx, cfg.y0, cfg.y1, cfg.ny);

    LinearElasticIsotropicMaterial matrix;
    matrix.set_parameter("E", cfg.E_m);
    matrix.set_parameter("nu", cfg.nu_m);
    matrix.set_name("Epoxy");
    mesh.add_material(&matrix);
    mesh.set_material("Epoxy");
    if (cohesive) {
        OPCohesiveMaterial coh_mat;
        coh_mat.set_parameter("sigma", cfg.coh_sigma);
        coh_mat.set_parameter("delta", cfg.coh_delta);
        coh_mat.set_parameter("beta", cfg.coh_beta);
        coh_mat.set_parameter("viscosity", cfg.coh_visc);
        coh_mat.set_name("Epoxy-Carbon");
        mesh.add_material(&coh_mat);
    }

    // Boundary conditions (PIGFEM4.6.1/Tests/Main.cpp:444-450)
    const double app_disp = (cfg.x1 - cfg.x0) * cfg.strain;
    BoundaryObject* boundary = problem->get_boundary();
    boundary->set_dirichlet_bcs_from_nodeset("right", 0, app_disp);
    boundary->set_dirichlet_bcs_from_nodeset("left", 0, 0.0);
    for (unsigned int d = 0; d < mesh.dim(); ++d) boundary->set_dirichlet_bc(0, d, 0);

    // Shape sensitivities of the right-edge load (Problem::addSensitivityFunction,
    // Problem::addShapeSensitivityParameter, Problem.cpp:836-861); Problem::init
    // builds the sensitivity solver (Problem.cpp:191-235)
    if (!cfg.sens.empty()) {
        SensitivityRightLoad fn;
        problem->addSensitivityFunction(&fn);
        for (const auto& p : cfg.sens) problem->addShapeSensitivityParameter((id_type)p.inc, p.name);
    }
    const double t_init0 = now_s();
    problem->init();
    const double t_init = now_s() - t_init0;

    Solver* solver = problem->get_solver();
    solver->set_dparameter("rel_tol", 1e-8);
    solver->set_dparameter("abs_tol", 1e-8);
    solver->set_dparameter("max_time_step", cfg.max_dt);
    solver->set_dparameter("min_time_step", cfg.min_dt);
    solver->set_dparameter("T_final", cfg.T_final);
    solver->set_iparameter("max_iter", cfg.max_iter);

    FILE* fp = fopen(argv[2], "wb");
    if (!fp) { fprintf(stderr, "cannot write %s\n", argv[2]); return 2; }
    Out o{fp};

    double t_asm_rep = 0.0;
    if (cfg.assemble_repeats > 0 && !cohesive) {
        problem->setup();
        Assembler* assem = problem->get_assembler();
        std::vector<double> each;
        for (int r = 0; r < cfg.assemble_repeats; ++r) {
            MatZeroEntries(solver->_K.ff); MatZeroEntries(solver->_K.fp);
            MatZeroEntries(solver->_K.pf); MatZeroEntries(solver->_K.pp);
            const double t0 = now_s();
            assem->assemble_linear(solver->_K);
            each.push_back(now_s() - t0);
            t_asm_rep += each.back();
        }
        o.d1("time.assemble_repeat_total", t_asm_rep);
        o.d("time.assemble_each", each);
        o.d1("time.init", t_init);
        o.i1("time.assemble_repeats", cfg.assemble_repeats);
        o.i1("mesh.n_elem_active", (int32_t)mesh.n_local_active_elem());
        fclose(fp);
        return 0;
    }

    // Per-load-step Newton statistics are collected by wrapping nothing: the
    // shim counts SNES iterations globally.
    const long snes0 = pgshim_snes_iterations();
    const double t_solve0 = now_s();
    problem->solve_problem();
    const double t_total_solve = now_s() - t_solve0;
#ifdef PG_GPU_DROPIN
    if (!cohesive) {
        SolverGPULinear* gs = dynamic_cast<SolverGPULinear*>(problem->get_solver());
        if (!gs || gs->status() != 0) {
            fprintf(stderr, "drop-in solve failed\n");
            return 3;
        }
        o.i1("gpu.iterations", gs->stats().iterations);
        o.d1("gpu.rel_residual", gs->stats().rel_residual);
    }
#endif

    // ---- mesh -------------------------------------------------------------
    std::vector<double> xy;
    for (id_type n = 0; n < mesh.n_local_nodes(); ++n) {
        Node* nd = mesh.get_node_local(n);
        xy.push_back((*nd)(0));
        xy.push_back((*nd)(1));
    }
    o.d("mesh.node_xy", xy);
    std::vector<double> exy;
    std::vector<int32_t> eedge, einc;
    for (id_type n = 0; n < mesh.n_local_enrich_nodes(); ++n) {
        Node* nd = mesh.get_enrich_node(n);
        exy.push_back((*nd)(0));
        exy.push_back((*nd)(1));
        auto e = mesh._enrich_node_to_edge[n];
        eedge.push_back((int32_t)e.first);
        eedge.push_back((int32_t)e.second);
        einc.push_back((int32_t)mesh._enrich_node_to_inclusion[n]);
    }
    o.d("mesh.enr_xy", exy);
    o.i("mesh.enr_edge", eedge);
    o.i("mesh.enr_inclusion", einc);
    o.i("mesh.node_detect", std::vector<int32_t>(mesh._node_detect.begin(), mesh._node_detect.end()));

    // element connectivity, material ids and the cut description
    std::vector<int32_t> conn, emat, cut_ptr(1, 0), cut_enr, child_ptr(1, 0), child_nodes, child_nodes_ptr(1, 0),
        child_mat, coh_ptr(1, 0), coh_nodes, coh_mat_id;
    std::vector<int32_t> is_cut;
    auto mat_index = [&](Material* m) -> int32_t { return m ? (int32_t)mesh.find_mat_number(m->get_name()) : -1; };
    for (id_type e = 0; e < mesh.n_local_elem(); ++e) {
        Elem* el = mesh.get_elem_local(e);
        for (id_type k = 0; k < el->n_nodes(); ++k) conn.push_back((int32_t)el->get_node(k)->get_id());
        emat.push_back((int32_t)mesh._elem_to_material[e]);
        is_cut.push_back(el->is_intersected() ? 1 : 0);
        if (el->is_intersected()) {
            for (id_type k = 0; k < el->n_enrich_nodes(); ++k)
                cut_enr.push_back((int32_t)(el->get_enrich_node(k)->get_id() - ENRICH_START));
            for (size_t c = 0; c < el->_int_elem_struct.size(); ++c) {
                for (auto v : el->_int_elem_struct[c]) child_nodes.push_back((int32_t)v);
                child_nodes_ptr.push_back((int32_t)child_nodes.size());
                child_mat.push_back(mat_index(el->_int_elem_mat[c]));
            }
            for (size_t c = 0; c < el->_coh_elem_struct.size(); ++c) {
                for (auto v : el->_coh_elem_struct[c]) coh_nodes.push_back((int32_t)v);
                coh_mat_id.push_back(mat_index(el->_coh_mat[c]));
            }
        }
        cut_ptr.push_back((int32_t)cut_enr.size());
        child_ptr.push_back((int32_t)child_mat.size());
        coh_ptr.push_back((int32_t)coh_mat_id.size());
    }
    o.i("mesh.conn", conn);
    o.i("mesh.elem_mat", emat);
    o.i("mesh.is_cut", is_cut);
    o.i("mesh.cut_enr_ptr", cut_ptr);
    o.i("mesh.cut_enr", cut_enr);
    o.i("mesh.child_ptr", child_ptr);
    o.i("mesh.child_nodes_ptr", child_nodes_ptr);
    o.i("mesh.child_nodes", child_nodes);
    o.i("mesh.child_mat", child_mat);
    o.i("mesh.coh_ptr", coh_ptr);
    o.i("mesh.coh_nodes", coh_nodes);
    o.i("mesh.coh_mat", coh_mat_id);
    std::vector<double> mat_E, mat_nu;
    for (auto* m : mesh._materials) {
        if (m->is_cohesive()) { mat_E.push_back(-1); mat_nu.push_back(-1); }
        else { mat_E.push_back(m->get_parameter("E")); mat_nu.push_back(m->get_parameter("nu")); }
    }
    o.d("mesh.mat_E", mat_E);
    o.d("mesh.mat_nu", mat_nu);

    // ---- DOFs -------------------------------------------------------------
    DofObject* dofs = problem->get_dofs();
    std::vector<int32_t> node_dofs, enr_dofs;
    for (id_type n = 0; n < mesh.n_local_nodes(); ++n)
        for (id_type d = 0; d < 2; ++d) node_dofs.push_back((int32_t)dofs->get_global_dof(n, d));
    for (id_type n = 0; n < mesh.n_local_enrich_nodes(); ++n)
        for (id_type d = 0; d < 2; ++d) enr_dofs.push_back((int32_t)dofs->get_global_dof(n + ENRICH_START, d));
    o.i("dof.node", node_dofs);
    o.i("dof.enr", enr_dofs);
    o.i1("dof.n_free", (int32_t)dofs->n_global_free_dofs());
    o.i1("dof.n_total", (int32_t)dofs->n_global_dofs());

    // ---- system -----------------------------------------------------------
    if (cfg.dump_K) {
        dump_mat(o, "K.ff", solver->_K.ff);
        dump_mat(o, "K.fp", solver->_K.fp);
        dump_mat(o, "K.pf", solver->_K.pf);
        dump_mat(o, "K.pp", solver->_K.pp);
    }
    dump_vec(o, "U.f", solver->_U.f);
    dump_vec(o, "U.p", solver->_U.p);
    dump_vec(o, "F.f", solver->_F_ext.f);
    dump_vec(o, "F.p", solver->_F_ext.p);
    if (!cohesive) {
        // Problem::compute_stress_strain at every volumetric quadrature point
        // (Problem.cpp:428-534), element by element, with the point's J W
        std::vector<int32_t> qp_count;
        std::vector<double> qp_strain, qp_stress, qp_jw;
        for (id_type e = 0; e < mesh.n_local_elem(); ++e) {
            Elem* el = mesh.get_elem_local(e);
            std::vector<std::vector<double>> strain, stress;
            problem->compute_stress_strain(strain, stress, el);
            qp_count.push_back((int32_t)strain.size());
            for (size_t q = 0; q < strain.size(); ++q) {
                for (int k = 0; k < 3; ++k) qp_strain.push_back(strain[q][k]);
                for (int k = 0; k < 3; ++k) qp_stress.push_back(stress[q][k]);
                qp_jw.push_back(mesh.get_J(e, q) * mesh.get_W(e, q));
            }
        }
        o.i("qp.count", qp_count);
        o.d("qp.strain", qp_strain);
        o.d("qp.stress", qp_stress);
        o.d("qp.jw", qp_jw);
    }
    if (cohesive) {
        SolverNonlinear* sn = dynamic_cast<SolverNonlinear*>(solver);
        dump_vec(o, "Pint.f", sn->_P_int.f);
        dump_vec(o, "Pint.p", sn->_P_int.p);
        // committed cohesive ISVs: delta_max for every cohesive quadrature point
        std::vector<int32_t> isv_elem, isv_qp;
        std::vector<double> isv_val;
        auto& iv = problem->get_internal_vars()->_internal_vars;
        for (size_t e = 0; e < iv.size(); ++e)
            for (size_t q = 0; q < iv[e].size(); ++q)
                if (!iv[e][q].empty()) {
                    isv_elem.push_back((int32_t)e);
                    isv_qp.push_back((int32_t)q);
                    isv_val.push_back(iv[e][q][0]);
                }
        o.i("isv.elem", isv_elem);
        o.i("isv.qp", isv_qp);
        o.d("isv.delta_max", isv_val);
        o.i1("snes.iterations", (int32_t)(pgshim_snes_iterations() - snes0));
    }
    if (!cfg.sens.empty()) {
        SensitivitySolver* ss = problem->_sensitivity_solver;
        o.d1("sens.f", ss->get_function_val(0));
        std::vector<double> g;
        for (size_t j = 0; j < cfg.sens.size(); ++j) g.push_back(ss->get_sensitivity(0, (id_type)j));
        o.d("sens.dfdp", g);
        o.i1("sens.adjoint", dynamic_cast<SensitivityAdjoint*>(ss) ? 1 : 0);
    }
    // the reference's writers on the final state (Writer_ASCII_VTK as
    // Problem::init builds it, Problem.cpp:246-249; WriterCohesiveOpenings)
    if (!cfg.vtk_out.empty()) {
        Writer_ASCII_VTK w(problem);
        w.store_mesh();
        w.write(cfg.vtk_out, cfg.T_final);
    }
    if (!cfg.openings_out.empty() && cohesive) {
        WriterCohesiveOpenings w(problem);
        w.store_mesh();
        w.write(cfg.openings_out, cfg.T_final);
    }
    o.d1("time.init", t_init);
    o.d1("time.assemble", problem->_assemble_time);
    o.d1("time.solve", problem->_solve_time);
    o.d1("time.total_solve", t_total_solve);
    o.d1("time.igfem_nodes", problem->_IGFEM_nodal_detection_time);
    o.d1("time.igfem_elems", problem->_IGFEM_element_detection_time);
    o.d1("time.igfem_enrich", problem->_IGFEM_enrichments_time);
    o.d1("time.ksp", pgshim_ksp_seconds());
    fclose(fp);
    return 0;
}
