/*
 * pigfem_b200.h -- C ABI of the B200 IGFEM assembly/solve path.
 *
 * Plain pointers and sizes only; every call returns an int status (0 = ok),
 * the way the reference's PETSc-touching calls return PetscErrorCode, and
 * none of them aborts.  A failed call leaves a message retrievable with
 * pg_last_error().  Streams are passed as opaque handles (cudaStream_t cast to
 * void*); NULL selects the context's own stream.
 *
 * Reference interfaces replaced (PIGFEM 4.6.1, paths relative to PIGFEM4.6.1/):
 *   Problem::init (IGFEM detection/enrichment, shape cache)  src/Problem.cpp:105-316
 *   Problem::setup / Solver::setup (DOFs, sparsity)          src/Problem.cpp:319-338, src/Solver.cpp:40-49,365-441
 *   Assembler::assemble_linear                               src/Assembler.cpp:48-89 (include/Assembler.h:41)
 *   Assembler::assemble_nonlinear                            src/Assembler.cpp:208-303 (include/Assembler.h:42-44)
 *   Assembler::assemble_new_load_step                        src/Assembler.cpp:554-663 (include/Assembler.h:51)
 *   PETScLinearKSPSolver::solve                              src/SolverLinear.cpp:91-162
 *   SolverNonlinear::solve / nonlinearStep (SNES Newton)     src/SolverNonlinear.cpp:111-397, src/SolverNonlinearSNES.cpp:182-241
 *   InternalVars::copy_data_in (ISV commit)                  src/InternalVars.cpp:65-85
 */
#ifndef PIGFEM_B200_H
#define PIGFEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define PG_OK 0
#define PG_ERR_ARG 1          /* invalid argument */
#define PG_ERR_MESH 2         /* IGFEM preprocessing failed (the reference would err_message + exit) */
#define PG_ERR_CUDA 3         /* CUDA runtime error */
#define PG_ERR_NOT_CONVERGED 4/* iteration budget exhausted (Krylov or Newton) */
#define PG_ERR_BREAKDOWN 5    /* Krylov breakdown (e.g. indefinite operator under CG) */
#define PG_ERR_STATE 6        /* call out of order (e.g. solve before assemble) */
#define PG_ERR_LIMIT 7        /* size beyond a documented maximum */

typedef struct pg_mesh pg_mesh;  /* host IGFEM mesh (opaque) */
typedef struct pg_ctx pg_ctx;    /* device state for one mesh (opaque) */

/* Cohesive laws.  PG_COH_OP: Ortiz-Pandolfi exponential law with linear
 * unloading and viscous regularisation, params {sigma_c, delta_c, beta,
 * viscosity, unused} (src/Material_OPCohesive.cpp:38-253, the reference's active law).
 * PG_COH_BILINEAR: bilinear penalty law, params {sigma_c, G_c, K_p, beta, eta}:
 * eta >= 0 adds the viscous traction eta * (delta_eff - delta_max) / dt while
 * the interface loads, the regularisation the OP law carries (0 = none). */
#define PG_COH_OP 0
#define PG_COH_BILINEAR 1

/* RVE description: the inputs the reference's driver builds through
 * Mesh::generate_mesh(TRI3, ...), Mesh::add_inclusion(Circle_Inclusion),
 * Mesh::add_material and BoundaryObject::set_dirichlet_bcs_from_nodeset
 * (Tests/Main.cpp:256, 310-450). */
typedef struct pg_rve_desc {
    int32_t nx, ny;                 /* structured TRI3 mesh, 2*nx*ny triangles */
    double x0, x1, y0, y1;          /* domain */
    int32_t n_inclusions;
    const double* inc_cx;           /* n_inclusions each */
    const double* inc_cy;
    const double* inc_r;
    const int32_t* inc_mat;         /* material index of each inclusion */
    int32_t n_materials;
    const double* mat_E;            /* linear elastic isotropic (material_lei.cpp:52-97) */
    const double* mat_nu;
    int32_t matrix_mat;             /* material of the background */
    int32_t plane_strain;           /* 1: plane strain (only mode of the configs), 0: plane stress */
    int32_t cohesive;               /* 1: inclusion interfaces carry cohesive elements */
    int32_t coh_law;                /* PG_COH_OP or PG_COH_BILINEAR */
    double coh_params[5];
    double strain;                  /* prescribed x-displacement of the right edge = (x1-x0)*strain */
} pg_rve_desc;

typedef struct pg_mesh_info {
    int32_t n_nodes;                /* regular + enrichment nodes */
    int32_t n_regular_nodes;
    int32_t n_enrichment_nodes;
    int32_t n_elements;
    int32_t n_cut_elements;
    int32_t n_cohesive_qp;
    int32_t n_dof;                  /* 2 * n_nodes */
    int32_t n_free_dof;
    int32_t n_blocks;               /* 2x2 blocks in the stiffness pattern (nnz = 4 * n_blocks) */
    int32_t n_moved_nodes;          /* nodes moved off an inclusion surface */
} pg_mesh_info;

/* ---- host preprocessing (Problem::init IGFEM steps + Problem::setup DOFs/sparsity) ---- */
int pg_mesh_build(const pg_rve_desc* rve, pg_mesh** out);
/* The same preprocessing on the GPU `device` (Mesh::analyze_nodes/detect_node,
 * src/Mesh.cpp:2676-2714,2838-2918; Tri3::detection, src/tri3.cpp:287-541;
 * Mesh::add_enrichments, src/Mesh.cpp:3038-3202; DofObject::distribute_dofs,
 * src/DofObject.cpp:241-386; Solver::preallocate_matrix, src/Solver.cpp:365-441):
 * node detection, cut templates, enrichment nodes in the reference's (edge,
 * inclusion) set order, edge-circle roots, DOF numbering and the block-CSR
 * pattern with its slot tables, one thread per node, element, edge or row.
 * The resulting mesh is bit for bit the one pg_mesh_build makes (the same
 * FP64 operations, each rounded on its own); nodes on an interface are moved
 * by the host in node order, as the reference moves them.  A grid edge cut by
 * two different inclusions returns PG_ERR_MESH (pg_mesh_build handles it). */
int pg_mesh_build_device(const pg_rve_desc* rve, int32_t device, pg_mesh** out);
int pg_mesh_info_get(const pg_mesh* m, pg_mesh_info* info);
/* Copies out host arrays (any pointer may be NULL):
 *   xy[2*n_nodes] node coordinates (x, y interleaved; regular then enrichment nodes)
 *   conn[3*n_elements], elem_mat[n_elements], elem_cut[n_elements] (-1 or cut index)
 *   ref_dof[n_dof]: the reference's global DOF number (free-first, DofObject.cpp:241-386) of
 *                   this library's DOF 2*node+d
 *   fixed[n_dof] (1 = Dirichlet), ubar[n_dof] prescribed values at load factor 1 */
int pg_mesh_export(const pg_mesh* m, double* xy, int32_t* conn, int32_t* elem_mat, int32_t* elem_cut,
                   int32_t* ref_dof, uint8_t* fixed, double* ubar);
/* Cut-element description: template id, enrichment node of each slot (12 per element, -1 unused),
 * child materials (4 per element, -1 unused), first cohesive quadrature point. */
int pg_mesh_export_cut(const pg_mesh* m, int32_t* cut_elem, int32_t* cut_tmpl, int32_t* cut_enr,
                       int32_t* cut_child_mat, int32_t* cut_coh_qp0);
/* 2x2-block CSR pattern: row_ptr[n_nodes+1], col[n_blocks]. */
int pg_mesh_export_pattern(const pg_mesh* m, int32_t* row_ptr, int32_t* col);
/* Cut templates: 80 int32 per template -- n_cut_edges, n_enr, n_child, n_coh,
 * cut_edge[6], enr_inc_node[6], child_n[4], child_mat_node[4], child_nodes[4][6],
 * coh_nodes[3][4], padding; returns the count in *n. */
int pg_template_table(int32_t* out, int32_t* n);
void pg_mesh_destroy(pg_mesh* m);

/* ---- device context (Solver::setup: matrix/vector preallocation on the GPU) ---- */
int pg_ctx_create(const pg_mesh* m, int32_t device, pg_ctx** out);
void pg_ctx_destroy(pg_ctx* c);
int pg_ctx_sync(pg_ctx* c);

/* Assembler::assemble_linear: K = sum over active elements (uncut: 4-point rule,
 * cut: sub-element quadrature with enrichment functions) in FP64, written into the
 * context's 2x2-block CSR (values 4 per block, row-major). */
int pg_assemble_linear(pg_ctx* c, void* stream);
/* Same call for callers that hold the inputs and want K on the host: copies node
 * coordinates xy_host[2*n_nodes] (nullable) host->device, assembles, copies the
 * 4*n_blocks FP64 values to k_host (nullable).  The drop-in for assemble_linear
 * filling a host PETSc matrix. */
int pg_assemble_linear_host(pg_ctx* c, const double* xy_host, double* k_host);
/* Assembler::assemble_nonlinear: residual vector f_int (want_f) and tangent K (want_K) at
 * the displacement U_dev[n_dof] (device pointer; NULL: the context's solution), load
 * step dt, writing trial cohesive state.  The trial state restarts from the committed
 * state on every call, as InternalVars::copy_data does (Assembler.cpp:235). */
int pg_assemble_nonlinear(pg_ctx* c, const double* U_dev, double dt, int32_t want_f, int32_t want_K, void* stream);
/* Problem::compute_stress_strain (Problem.cpp:428-534) at every volumetric quadrature point,
 * element by element in the reference's point order (uncut: the 4 points of the Tri3 rule;
 * cut: each integration child's points in template order), at the displacement U_dev
 * (device pointer; NULL: the context's solution).  Outputs (each nullable):
 *   points_host[7*n_points]  per point: strain xx, yy, xy (engineering shear), stress xx, yy, xy
 *                            (plane strain, D eps), J W.  A point of zero weight (a collapsed
 *                            integration child) has NaN strain and stress, as in the reference.
 *   n_points                 the number of volumetric points
 *   elem_point_off[n_elem+1] first point of each element
 *   mean[7]                  J W-weighted volume averages of strain (3) and stress (3), then the
 *                            total J W (the homogenised response; zero-weight points skipped),
 *                            reduced on the device in a fixed order (bit-reproducible).
 * With points_host and mean both NULL only the counts and offsets are returned. */
int pg_stress_strain(pg_ctx* c, const double* U_dev, double* points_host, int64_t* n_points,
                     int32_t* elem_point_off, double* mean);
/* Writer_ASCII_VTK::write (Writer_ASCII_VTK.cpp, Writer_VTK.cpp:164-336, 639-911): the legacy
 * ASCII VTK file of the context's state at time t -- nodes (regular, then enrichment), cells
 * (uncut elements; integration children in place of cut ones), displacement and external
 * force per node (enrichment nodes: parent-edge interpolation plus their own value), and per
 * cell the reference's material number, partition 0, the means of strain and stress over its
 * quadrature points and the von Mises stress.  External force: zero on free DOFs, the
 * reaction on prescribed ones -- K U, formed here, for a linear mesh (this overwrites the
 * context's internal-force vector); for a cohesive mesh the internal force of the last
 * residual assembly (the Newton driver leaves the accepted state of its last load step). */
int pg_write_vtk(pg_ctx* c, const char* path, double t);
/* WriterCohesiveOpenings::write (WriterCohesiveOpenings.cpp:39-197): one CSV line per
 * cohesive sub-element, "inclusion,theta,delta_t/delta_c,delta_n/delta_c" at its midpoint,
 * sorted, at precision 16 (delta_c: the Ortiz-Pandolfi law's; 2 G_c / sigma_c for the
 * bilinear law).  PG_ERR_ARG on a mesh without a cohesive interface. */
int pg_write_cohesive_openings(pg_ctx* c, const char* path);
/* Assembler::assemble_new_load_step: prescribed values = t_frac * ubar. */
int pg_new_load_step(pg_ctx* c, double t_frac);
/* InternalVars::copy_data_in: committed cohesive state <- trial state. */
int pg_commit_isv(pg_ctx* c);

/* Device pointers to the context's arrays (valid until pg_ctx_destroy). */
int pg_ctx_device_arrays(pg_ctx* c, double** K, double** U, double** F_int, double** isv_committed,
                         double** isv_trial);

/* ---- solvers ---- */
#define PG_KRYLOV_CG 0
#define PG_KRYLOV_GMRES 1
#define PG_KRYLOV_MINRES 2      /* symmetric indefinite tangents; |diag| Jacobi preconditioner */
#define PG_PREC_JACOBI 0
#define PG_PREC_BLOCK_JACOBI 1
#define PG_PREC_NONE 2
#define PG_PREC_MG 3               /* one geometric multigrid V-cycle over the structured background grid
                                      (Galerkin coarse operators, damped block-Jacobi smoothing); with
                                      PG_PRECISION_MIXED the V-cycle runs in FP32 inside the FP64 Krylov loop */
#define PG_PRECISION_FP64 0        /* plain FP64 Krylov */
#define PG_PRECISION_MIXED 1       /* Jacobi preconditioners: Krylov on the FP32-stored matrix (FP64 vectors
                                      and dots) inside FP64 iterative refinement on the FP64 residual;
                                      PG_PREC_MG: FP32 V-cycle preconditioning an FP64 Krylov solve */

typedef struct pg_solver_cfg {
    int32_t krylov;                 /* PG_KRYLOV_* */
    int32_t precond;                /* PG_PREC_* */
    int32_t precision;              /* PG_PRECISION_* */
    double rtol;                    /* relative residual target of the linear solve (FP64 residual) */
    int32_t max_iter;               /* Krylov iteration budget (total over refinements) */
    double inner_rtol;              /* mixed: FP32 inner solve tolerance per refinement */
    int32_t max_refine;             /* mixed: refinement budget */
    int32_t gmres_restart;
    int32_t check_every;            /* host residual check cadence (iterations per captured graph) */
    int32_t inclusion_modes;        /* PG_PREC_MG on cohesive meshes: 1 adds the inclusions' rigid motions
                                       (3 per inclusion) as a coarse space (default 0) */
    int32_t deterministic;          /* 1 (default): every Krylov dot product is summed in a fixed order (block
                                       partials added in block order by the grid's last block), so a solve is
                                       bit-reproducible run to run; 0: block partials are added with atomics,
                                       order-dependent in the last bits, a few microseconds less per reduction */
} pg_solver_cfg;

typedef struct pg_solve_stats {
    int32_t iterations;             /* Krylov iterations */
    int32_t refinements;            /* FP64 refinement steps (mixed) */
    double rel_residual;            /* final FP64 ||r_f|| / ||r_f(0)|| */
    double seconds;                 /* device time of the solve */
    int32_t newton_iterations;
    int32_t status;
} pg_solve_stats;

void pg_solver_cfg_default(pg_solver_cfg* cfg);
/* PETScLinearKSPSolver::solve: prescribed U_p = ubar (load factor 1), rhs = -K_fp U_p,
 * K_ff U_f = rhs, reactions F_p = K_pf U_f + K_pp U_p.  Assembles K first if needed. */
int pg_solve_linear(pg_ctx* c, const pg_solver_cfg* cfg, pg_solve_stats* stats);

/* ---- nonlinear load stepping (cohesive RVEs) ---- */
#define PG_PREDICT_ZEROTH 0   /* keep the last converged free DOFs (the reference, SolverNonlinear.cpp:254-267) */
#define PG_PREDICT_LINEAR 1   /* extrapolate linearly in the load factor */
#define PG_PREDICT_GIVEN 2    /* the caller set U before the step */
#define PG_PREDICT_LEARNED 3  /* linear extrapolation corrected by the attached MLP; the linear
                                 extrapolation is kept whenever it starts from a smaller residual */

typedef struct pg_newton_cfg {
    int32_t n_steps;                /* equal load steps to T_final */
    double T_final;
    double rtol, atol, stol;        /* SNES defaults: 1e-8, 1e-50, 1e-8 */
    int32_t max_it;                 /* Newton iterations per step (SNES default 50) */
    int32_t precision;              /* linear solves: PG_PRECISION_FP64 or PG_PRECISION_MIXED */
    int32_t precond;
    double lin_rtol;                /* floor of the Krylov forcing term */
    double inner_rtol;              /* mixed: FP32 inner tolerance */
    int32_t lin_max_iter;
    int32_t max_repeat;             /* load-step repeats with dt *= 0.25 (reference: 20) */
    int32_t predictor;              /* PG_PREDICT_* */
    int32_t rtol_base;              /* PG_RTOL_BASE_*: which residual rtol is relative to */
    int32_t inclusion_modes;        /* as in pg_solver_cfg (default 0) */
    double t_start, t_stop;         /* pg_solve_nonlinear steps the load fraction from t_start (the current U and
                                       committed state are converged there) to t_stop; defaults 0 and 1 */
    int32_t deterministic;          /* as in pg_solver_cfg (default 1): with 1 a load path is bit-reproducible */
} pg_newton_cfg;
/* rtol relative to the residual of the step's own predictor (SNES, the reference) */
#define PG_RTOL_BASE_PREDICTOR 0
/* rtol relative to the residual of the zeroth-order predictor (the last converged
 * U_f with the new prescribed values): one target per load step whatever the
 * predictor, so predictors are compared at the same accuracy */
#define PG_RTOL_BASE_ZEROTH 1

typedef struct pg_step_stats {
    double t_frac, dt;
    int32_t newton_its, krylov_its, gmres_fallbacks, repeats;  /* pg_solve_nonlinear: summed over all attempts */
    double res0, res;               /* FP64 ||r|| of the predictor and at the end */
    int32_t reason;                 /* SNES-style: 2 abs, 3 rel, 4 step; <0 diverged */
    double seconds;                 /* pg_newton_load_step: device time of the step; pg_solve_nonlinear: wall time
                                       of the load step from its predictor to acceptance, every attempt included */
    int32_t predictor_used;         /* PG_PREDICT_* actually used for this step */
    double res_linear, res_learned; /* initial residuals of both candidates (learned predictor only) */
    double res_base;                /* the residual rtol was relative to */
    double blend;                   /* learned predictor: the blend g of the step's learned candidate (0: linear,
                                       1: quadratic extrapolation); -1 when no learned candidate was formed */
} pg_step_stats;

void pg_newton_cfg_default(pg_newton_cfg* cfg);
/* SolverNonlinearSNES::nonlinearStep for one load step at load factor t_frac with
 * step dt (viscous regularisation); the trial cohesive state is left for pg_commit_isv. */
int pg_newton_load_step(pg_ctx* c, double t_frac, double dt, const pg_newton_cfg* cfg, pg_step_stats* stats);
/* SolverNonlinear::solve: equal load steps with the reference's step cutting on failure;
 * commits the cohesive state after every converged step.  Writes up to max_records
 * step records. */
int pg_solve_nonlinear(pg_ctx* c, const pg_newton_cfg* cfg, pg_step_stats* per_step, int32_t max_records,
                       int32_t* n_records);

/* ---- learned Newton warm start: per-node MLP (no counterpart in the reference) ----
 * 16 -> 64 -> 64 -> 16 ReLU network (2 outputs used), BF16 weights/activations on the
 * tcgen05 tensor cores with FP32 accumulation; parameters are FP32 masters laid out
 * W1[64x16], b1[64], W2[64x64], b2[64], W3[16x64], b3[16] (row = output). */
typedef struct pg_mlp pg_mlp;
int pg_mlp_create(int32_t device, uint64_t seed, pg_mlp** out);
void pg_mlp_destroy(pg_mlp* m);
int32_t pg_mlp_param_count(void);
int pg_mlp_params(pg_mlp* m, float* host, int32_t set);     /* set=1: upload (resets Adam), 0: download */
int pg_mlp_grads(pg_mlp* m, float* host);                  /* gradient of the last pg_mlp_gradient */
int pg_mlp_forward(pg_mlp* m, const float* X_dev, int32_t n, float* Y_dev, void* stream);
int pg_mlp_gradient(pg_mlp* m, const float* X_dev, const float* T_dev, int32_t n, double* loss_host);
int pg_mlp_adam(pg_mlp* m, float lr);
int pg_mlp_train(pg_mlp* m, const float* X_dev, const float* T_dev, int32_t n, int32_t epochs, int32_t batch,
                 float lr, double* loss_hist);
/* Self-test of the kernels' bounded completion waits (the failure path the
 * reference has no counterpart for): one forward tile whose first GEMM is
 * not issued, so its mbarrier is never signalled and the wait gives up after
 * `polls` polls with nothing in flight.  Returns PG_ERR_STATE ("timed out");
 * the network and the device stay usable. */
int pg_mlp_wait_selftest(pg_mlp* m, int32_t polls);

/* Learned-predictor plumbing (device pointers).  The history of a step: the
 * converged states at t_n, t_{n-1}, t_{n-2}, the steps dt_n and dt_{n-1} that
 * led to the first two, the coming step dt, the load fraction at t_n + dt and
 * the step's prescribed displacement increment.  The prediction is
 *   U = U_n + (dt/dt_n) d_n + g c,  d_n = U_n - U_{n-1},
 *   c = dt (dt + dt_n) / (dt_n + dt_{n-1}) (d_n/dt_n - d_{n-1}/dt_{n-1})
 * per node, with one blend g = sum |c_i|^2 (1 + y_i) / sum |c_i|^2 of the
 * linear (g = 0) and quadratic (g = 1) extrapolations, y_i the network's
 * output for node i clamped to [-1, 0].  Features: 16 floats per node;
 * targets and outputs: 2 floats per node (both y). */
typedef struct pg_pred_history {
    const double* U_n;
    const double* U_nm1;
    const double* U_nm2;
    const double* isv_nm1;          /* committed delta_max at t_{n-1} (NULL: no damage-rate feature); the
                                       context's committed state is taken as t_n's */
    double dt_n, dt_nm1, dt;
    double t_frac;
    double s_inc;
} pg_pred_history;
int pg_predictor_features(pg_ctx* c, const pg_pred_history* h, float* X_dev);
/* targets of the step that reached U_np1 (training data) */
int pg_predictor_targets(pg_ctx* c, const pg_pred_history* h, const double* U_np1, float* T_dev);
/* U_dev (free DOFs) = the prediction with g scaled by `scale` (Y_dev NULL: the linear extrapolation) */
int pg_predictor_apply(pg_ctx* c, const pg_pred_history* h, const float* Y_dev, double scale, double* U_dev);
/* attaches a network for PG_PREDICT_LEARNED (NULL detaches; the context does not own it) */
int pg_ctx_attach_mlp(pg_ctx* c, pg_mlp* m);

/* ---- host copies (tests, parity, output) ---- */
int pg_get_matrix(pg_ctx* c, double* vals_host);         /* 4*n_blocks */
int pg_get_vector(pg_ctx* c, int32_t which, double* out); /* which: 0=U, 1=F_int, 2=reaction/residual work */
int pg_set_vector(pg_ctx* c, int32_t which, const double* in);
int pg_get_isv(pg_ctx* c, int32_t committed, double* out);/* n_cohesive_qp delta_max values */
int pg_set_isv(pg_ctx* c, int32_t committed, const double* in);
/* Device time of the last assembly, from CUDA events recorded on the assembly stream
 * while timing is enabled.  enable = 1 (split): ms_rows = the triangle kernel, ms_cut =
 * from its end to the end of the pass (the cut elements' kernels and the fold); the event
 * between them keeps the cut kernels from starting in the triangle kernel's last wave.
 * enable = 2 (whole pass): ms_rows = the pass, ms_cut = 0, with the cut kernels launched
 * as programmatic dependents of the triangle kernel as in untimed passes.  0: off.  The
 * values returned are those of the mode in force during the last assembly; pass NULLs
 * to only switch modes. */
int pg_assembly_timing(pg_ctx* c, int32_t enable, float* ms_rows, float* ms_cut);

/* ---- shape sensitivity ----
 * SensitivityAdjoint::solveProblem with SensitivityRightLoad (src/SensitivityAdjoint.cpp:23-63,
 * src/SensitivityRightLoad.cpp:32-125) and the shape parameters of
 * Problem::addShapeSensitivityParameter (src/Problem.cpp:856-861; Circle_Inclusion's
 * "X", "Y", "R": src/InclusionCircle.cpp:176-227; the derivative of the element
 * force: src/SensitivityShapeParameterStructural.cpp:18-230).
 * At the context's current equilibrium U (solve first): f = the sum of the right
 * edge's x reactions / height (SensitivityRightLoad::evaluate), and df/dd for each
 * parameter d = (inclusion[p], kind[p]) from one adjoint solve (cfg: CG/GMRES, any
 * preconditioner) and the analytic shape derivative of every cut element's internal
 * force along the parameter's velocity field.  dfdp: n_params values (NULL allowed).
 * PG_ERR_ARG for an inclusion out of range or an unknown kind. */
#define PG_SHAPE_X 0   /* centre x */
#define PG_SHAPE_Y 1   /* centre y */
#define PG_SHAPE_R 2   /* radius */
int pg_sensitivity_shape(pg_ctx* c, const pg_solver_cfg* cfg, int32_t n_params, const int32_t* inclusion,
                         const int32_t* kind, double* f, double* dfdp, pg_solve_stats* adjoint_stats);
/* C_11 = f / applied strain and dC_11/dr_i for the radius of every inclusion
 * (dc11_dr: n_inclusions values, NULL allowed).  h_rel = 0: the analytic derivative
 * (pg_sensitivity_shape); h_rel > 0: a central difference of each cut element's
 * internal force under moves of its enrichment nodes by +-h_rel r_i along the
 * velocity (a cross-check of the analytic path, O(h^2) accurate). */
int pg_sensitivity_c11(pg_ctx* c, const pg_solver_cfg* cfg, double h_rel, double* c11, double* dc11_dr,
                       pg_solve_stats* adjoint_stats);

/* ---- autotuning of the assembly launch shapes ----
 * No counterpart in the reference.  Times every launch shape of the two
 * assembly stages on this context's mesh (L2 flushed before each launch,
 * `reps` launches each) and keeps the fastest of each for later assemblies:
 * ms_tri[5] = the row-tile triangle kernel gathering over 32 / 64 consecutive
 * node rows per CTA, each with one CTA per tile / a persistent grid, then the
 * structured-grid kernel (one thread per regular node row; the fastest of 128
 * and 256 threads per CTA, each with one CTA per tile or a persistent grid
 * that stages the next tile with asynchronous copies while forming the
 * current one; 0 if the mesh is not made of structured grids);
 * ms_cut[3] = the cut elements' work (cohesive points, quadrature rows and
 * blocks, fold) with 2 / 4 / 8 warps per CTA of the cut-element kernel (NULL
 * allowed); then, with the structured-grid kernel, whole passes of both its
 * variants with the cut elements' kernels after it or beside it
 * (pg_ctx_cut_overlap).  K is left to be reassembled. */
int pg_ctx_autotune(pg_ctx* c, int32_t reps, float* ms_tri, float* ms_cut);
/* the launch shapes in use, and setting them by hand (tile 32 or 64 node rows per CTA of the
 * row-tile kernel, or 128 / 256 threads per CTA of the structured-grid kernel; persistent 0/1
 * for either; warps 2/4/8 per CTA of the cut elements' kernel) */
int pg_ctx_tuning(pg_ctx* c, int32_t* tri_tile_nodes, int32_t* tri_persistent, int32_t* cut_warps);
int pg_ctx_set_tuning(pg_ctx* c, int32_t tri_tile_nodes, int32_t tri_persistent, int32_t cut_warps);
/* With the structured-grid kernel: 0 runs the cut elements' kernels after it on the same
 * stream; 1 or 2 runs them beside it on a second stream, the persistent grid kernel leaving
 * them that many CTA slots per SM.  The autotuner times every combination with both grid
 * variants on whole passes.  set < 0 only reads; get may be NULL. */
int pg_ctx_cut_overlap(pg_ctx* c, int32_t set, int32_t* get);

/* ---- batches of independent linear-elastic RVEs ----
 * No counterpart in the reference, which solves one RVE per run
 * (Problem::solve_problem, src/Problem.cpp:400-418).  A batch is the
 * block-diagonal union of n_rve meshes (built by pg_mesh_build, any sizes):
 * one launch of each assembly kernel covers all of them (assemble through
 * pg_batch_context + pg_assemble_linear), and pg_batch_solve runs CG with
 * per-RVE step lengths and per-RVE stopping (rtol relative to each RVE's own
 * right-hand side), preconditioned by block Jacobi or by one V-cycle over the
 * union of the RVEs' multigrid hierarchies (PG_PREC_MG; FP32 cycle under
 * PG_PRECISION_MIXED).  The CG iterations run as CUDA graphs. */
typedef struct pg_batch pg_batch;
int pg_batch_create(const pg_mesh* const* meshes, int32_t n_rve, int32_t device, pg_batch** out);
void pg_batch_destroy(pg_batch* b);
/* the merged system as a context: assembly, timing and host copies work on it */
pg_ctx* pg_batch_context(pg_batch* b);
/* host seconds of pg_batch_create's phases (7 values): recording the RVEs'
 * grids, merging the meshes (in parallel on the host's cores, read in place),
 * the context's uploads, grid tiles, cut-element tables and fold order (built
 * on the GPU), and the multigrid hierarchy */
int pg_batch_setup_times(const pg_batch* b, double* seconds);
/* first node / element of each RVE in the merged system (n_rve + 1 entries each), multigrid depth per RVE */
int pg_batch_info(const pg_batch* b, int32_t* node_offset, int32_t* element_offset, int32_t* depth);
/* solves every RVE (prescribed values at load factor 1); per_rve: n_rve records or NULL; total: worst of all */
int pg_batch_solve(pg_batch* b, const pg_solver_cfg* cfg, pg_solve_stats* per_rve, pg_solve_stats* total);
/* the RVE's displacements in its own mesh's DOF order (2 * its node count) */
int pg_batch_get_solution(pg_batch* b, int32_t rve, double* U_host);

/* ---- solve without device allocation ----
 * No counterpart in the reference.  For callers that cannot let this library
 * allocate device memory (a host framework that owns every device buffer
 * through its own allocator or budget, code where an allocation is not
 * permitted, foreign-language bindings that hold only pointers): block-Jacobi
 * PCG on a caller-owned 2x2-block CSR system of at most PG_STATIC_MAX_NODES
 * nodes (2 DOFs each, DOF 2*node+d), solving mask(K) x = mask(b) on the DOFs
 * with fixed[dof] == 0 and writing x = 0 on the others.  All pointers are
 * device pointers the caller owns (row_ptr n_nodes+1, col and 4 values per
 * block, fixed/b/x 2*n_nodes); stats is host memory.  The Krylov vectors live
 * in one fixed array of about 3 MiB in the library's device image, held on
 * every GPU that loads the library until exit: the first call on a device
 * (with that device current) looks its address up, so make that first call
 * before any stream capture; every call shares the array, so calls that
 * overlap on the GPU race and must be serialised.  Returns PG_ERR_LIMIT for
 * more than PG_STATIC_MAX_NODES nodes and never calls cudaMalloc or cudaFree.
 * stream: cudaStream_t cast to void* (NULL = legacy default stream). */
#define PG_STATIC_MAX_NODES 32768
int pg_pcg_solve_static(int32_t n_nodes, const int32_t* row_ptr, const int32_t* col, const double* K,
                        const uint8_t* fixed, const double* b, double* x, double rtol, int32_t max_iter,
                        void* stream, pg_solve_stats* stats);

const char* pg_last_error(void);
const char* pg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PIGFEM_B200_H */
