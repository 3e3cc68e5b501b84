// Internal device-side state of the B200 IGFEM path (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "igfem_host.h"
#include "pigfem_b200.h"

struct pg_mesh {
    pgb::HostMesh m;
};

namespace pgb {

// cudaMemcpy from pageable host memory and cudaMemset run on the legacy
// default stream, which the library's non-blocking streams do not wait for,
// and may return before the data is in place (a pageable copy returns once
// the data is staged).  Set-up code copies and fills through these two, which
// wait until the data is written, so that a kernel launched next on any
// stream reads it.
inline cudaError_t h2d_sync(void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}
inline cudaError_t fill_sync(void* dst, int value, size_t bytes) {
    cudaError_t e = cudaMemset(dst, value, bytes);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}

// Runs fn(i) for i in [0, n) on the host's cores, in chunks of `grain`
// consecutive indices (each index exactly once; fn must not throw).
template <class F>
void parallel_for(long long n, long long grain, F&& fn) {
    if (n <= 0) return;
    const long long chunks = (n + grain - 1) / grain;
    const int T = (int)std::min<long long>(chunks, std::max(1u, std::min(std::thread::hardware_concurrency(), 32u)));
    if (T <= 1) {
        for (long long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<long long> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t)
        pool.emplace_back([&] {
            for (long long ch; (ch = next.fetch_add(1)) < chunks;)
                for (long long i = ch * grain, e = std::min(n, i + grain); i < e; ++i) fn(i);
        });
    for (auto& th : pool) th.join();
}

// Cohesive law parameters on the device.
struct DevCohLaw {
    int law;          // PG_COH_OP / PG_COH_BILINEAR
    double p[5];
};

// Template table entry as the cut-element kernel reads it (constant memory).
// Cut elements are integrated by one kernel instance per size class: local
// node count (3 + enrichment slots) at most kCutClassNl[k].
constexpr int kCutClasses = 4;
constexpr int kCutClassNl[kCutClasses] = {5, 7, 11, 15};
constexpr int kCutNodeStride = 16;
constexpr int kCohRowDoubles = 10;  // row of a cohesive Gauss point (k_coh_points)

struct DevTemplate {
    int n_enr, n_child, n_coh, pad;
    int child_n[kMaxChildren];
    int child_type[kMaxChildren];
    int child_nodes[kMaxChildren][kMaxChildNodes];
    int coh_nodes[kMaxCoh][4];
};

constexpr int kMaxChildQ = 24;
struct DevChildQuad {
    int nq, nn, pad0, pad1;
    double w[kMaxChildQ];
    double N[kMaxChildQ * kMaxChildNodes];
    double dN[kMaxChildQ * kMaxChildNodes * 2];
};

struct MgHierarchy;

// Uncut-triangle assembly tiling (k_assemble_tri) and the per-block map that
// tells each 2x2 block which staged (node, triangle) entries of its CTA
// contribute to it.  Map word of a block: bits 0-9 entry e0 and bits 10-11
// its vertex t0 that is the block's column node, bits 12-21 / 22-23 the
// second entry, bits 24-25 the count (0-2); kTriMapDiag marks the diagonal
// block, kTriMapSlow a block whose entries do not fit the word (evaluated
// from global memory).  Entries are numbered from the CTA's first entry, so
// the map depends on the tile size: one map per tile size the autotuner may
// pick (kTriTileSizes node rows per CTA, 2 threads and 8 staged entries per row).
constexpr int kTriTileVariants = 2;
constexpr int kTriTileSizes[kTriTileVariants] = {32, 64};
constexpr int kTriMapDiag = 1 << 28;
constexpr int kTriMapSlow = 1 << 29;
void build_tri_map(const HostMesh& hm, int tile_nodes, std::vector<int>& map);
bool grid_pattern_ok(const HostMesh& hm);  // block rows laid out as the structured-grid kernel assumes
constexpr int kGridTileCols = 64;          // node columns per structured-grid tile
// Autotuned launch shapes of the assembly kernels (pg_ctx_autotune):
// the structured-grid kernel's CTA size, or (meshes without one grid) the
// row-tile kernel's tile size and persistent grid (CTAs walk the tiles) or
// one CTA per tile, and the warps per CTA of the cut-element kernel.
struct AsmTuning {
    int tri_grid = 1;      // 1: the structured-grid kernel (when the mesh has one grid)
    int grid_block = 256;  // its threads per CTA: 128 or 256
    int tri_variant = 1;   // otherwise: index into kTriTileSizes
    int tri_persistent = 0;
    int cut_warps = 4;     // 2, 4 or 8
    // with the structured-grid kernel: 0 runs the cut elements' kernels after
    // it on the same stream; 1 or 2 runs them beside it on a second stream (the
    // persistent grid kernel leaving them that many CTA slots per SM)
    int cut_overlap = 0;
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    HostMesh hm;                       // host copy (sizes, maps, export)
    int n_nodes = 0, n_reg = 0, n_elem = 0, n_cut = 0, n_blocks = 0, n_dof = 0, n_coh_qp = 0;
    DevCohLaw coh{};
    // mesh
    double* x = nullptr;
    double* y = nullptr;
    int4* elem4 = nullptr;             // n0, n1, n2, material
    int* row_ptr = nullptr;
    int* col = nullptr;
    int* diag = nullptr;
    int* ne_ptr = nullptr;
    int* ne_list = nullptr;
    int* tri_map[kTriTileVariants] = {};  // one word per block per tile size (see kTriMapDiag)
    AsmTuning tuning;
    int* grid_emat = nullptr;          // structured meshes: material per element, -1 for cut elements
                                       // (set only where the structured-grid kernel applies)
    int4* grid_rves = nullptr;         // per grid block: nx, ny, first node, first element
    int4* grid_tiles[2] = {};          // per tile of 2 / 4 node rows: grid block, I0, J0
    int n_grid_tiles[2] = {0, 0};
    double* dmat = nullptr;            // 3 per material: D11, D12, D33
    // cut elements, grouped by size class (kCutClassNl), in that order
    int* cut_nodes = nullptr;          // kCutNodeStride per element: 3 parent nodes, then enrichment slots, -1 unused
    int* cut_tmpl = nullptr;
    int* cut_child_mat = nullptr;      // kMaxChildren per element
    int* cut_coh_qp0 = nullptr;        // first cohesive quadrature point (mesh numbering)
    // quadrature rows of the cut elements ({w det, d11, d12, d33, (gx, gy) per
    // local function}, 4 + 2 NL doubles for size class NL, point-major per
    // element), formed from one record per point (build_cut_points): in
    // shared memory by k_cut_elems at every assembly, and in global memory by
    // k_cut_points for the stress recovery; per element (class order) its
    // first row's offset
    double* cut_rows = nullptr;        // (stress recovery only, allocated on its first use)
    long long cut_rows_len = 0;
    long long* cut_row_off = nullptr;
    int* cut_pts = nullptr;
    int n_cut_pts = 0;
    int* cut_pt_off = nullptr;         // per element (class order) its first point record, then the total
    // the widest span of rows (doubles) that one CTA of k_cut_elems forms in
    // shared memory, per size class and CTA size (2, 4, 8 warps)
    int cut_span[4][3] = {};
    int* cut_slot_ptr = nullptr;
    int* cut_slot = nullptr;           // (3 + n_enr)^2 block slots per element
    int cut_class_off[5] = {0, 0, 0, 0, 0};
    // deterministic assembly of the cut elements: pair blocks (4 FP64) in
    // fold order and residual terms (2 FP64) in node order, each slot-table
    // entry's positions there, and the runs the folds sum
    double* cut_ke = nullptr;
    double* cut_fe = nullptr;
    int* cut_kpos = nullptr;
    int* cut_fpos = nullptr;
    long long* fold_K_slot = nullptr;  // slot << 1 | cut_only
    int* fold_K_ptr = nullptr;
    int n_fold_K = 0;
    // slots with one cut contribution take it straight from k_cut_elems: per
    // slot-table entry slot << 1 | cut_only for those, -2 - (fold position)
    // for the others, -1 without a K slot; the runs of two or more (their key
    // and their range of ke) are left to k_fold_K
    long long* cut_kdir = nullptr;
    long long* fold_Km_slot = nullptr;
    int2* fold_Km_rng = nullptr;
    int n_fold_Km = 0;
    int* fold_f_node = nullptr;        // node << 1 | cut_only
    int* fold_f_ptr = nullptr;
    int n_fold_f = 0;
    int* coh_rec = nullptr;            // per cohesive point: class-ordered element << 8 | sub-element << 1 | point
    double* coh_rows = nullptr;        // per cohesive point: kCohRowDoubles FP64 (k_coh_points)
    MgHierarchy* mg = nullptr;         // multigrid hierarchy, built at the first multigrid solve
    // system
    double* K = nullptr;               // 4 * n_blocks
    float* Kf = nullptr;               // FP32 copy for mixed precision
    uint8_t* fixed = nullptr;          // n_dof
    double* ubar = nullptr;            // n_dof
    double* U = nullptr;               // n_dof (full vector incl. prescribed)
    double* F = nullptr;               // n_dof internal force / work
    double* isv_c = nullptr;           // committed delta_max
    double* isv_t = nullptr;           // trial delta_max
    // solver work (FP64)
    double* r = nullptr;
    double* z = nullptr;
    double* p = nullptr;
    double* q = nullptr;
    double* dx = nullptr;
    double* minv = nullptr;            // 4 per node: inverse of the (masked) diagonal 2x2 block or Jacobi
    // solver work (FP32)
    float* rf = nullptr;
    float* zf = nullptr;
    float* pf = nullptr;
    float* qf = nullptr;
    float* xf = nullptr;
    float* minvf = nullptr;
    double* b = nullptr;               // right-hand side of the current Krylov solve
    double* res = nullptr;             // Newton residual
    double* Ut = nullptr;              // Newton trial displacement
    double* Uprev = nullptr;           // last converged displacement
    double* Uold = nullptr;            // the one before (linear extrapolation predictor)
    double* Uold2 = nullptr;           // and the one before that (learned predictor's history)
    double* isv_prev = nullptr;        // committed delta_max one step back (learned predictor's history)
    double* V = nullptr;               // GMRES basis, (gm + 1) * n_dof, allocated on first use
    int gm = 0;
    double* hbuf = nullptr;            // GMRES multi-dot results (64)
    double* xi = nullptr;              // inner correction of the mixed-precision refinement
    double* mw = nullptr;              // MINRES direction buffers (2 * n_dof)
    // learned warm start
    pg_mlp* mlp = nullptr;             // attached network (not owned)
    int* nq_ptr = nullptr;             // node -> cohesive quadrature points
    int* nq_list = nullptr;
    float* featX = nullptr;            // 16 features per node
    float* featY = nullptr;            // 2 outputs per node
    double* scal = nullptr;            // device scalars
    double* red_ws = nullptr;          // deterministic grid-sum workspace (grid_add)
    double* red_active = nullptr;      // red_ws, or null while a solve sums with atomics (cfg.deterministic 0)
    int* iflags = nullptr;             // device flags
    double* h_scal = nullptr;          // pinned host mirror
    int* h_iflags = nullptr;
    bool assembled = false;
    double t_frac = 1.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // events bracketing the two assembly kernels of the last assembly (rows, cut)
    cudaEvent_t ea0 = nullptr, ea1 = nullptr, ea2 = nullptr;
    // second stream: the cut elements' quadrature rows are formed on it while
    // the structured-grid kernel runs (fork / join events)
    cudaStream_t aux = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    bool timing = false;
    bool timing_split = false;         // an event between the triangle kernel and the cut kernels too
    // stress/strain recovery (stress_prepare, on first use): per element its
    // first volumetric quadrature point, the cut flags, class order -> mesh
    // element, class offsets, and 7 FP64 per point of output
    int* qp_off = nullptr;
    int* qp_elem_cut = nullptr;
    int* qp_cut_elem = nullptr;
    int* qp_class_off = nullptr;
    double* qp_out = nullptr;
    long long n_qp_total = 0;
    // host seconds of the set-up phases of ctx_create: uploads of the mesh,
    // grid tiles, cut-element tables and point records, fold order
    double setup_s[4] = {0, 0, 0, 0};
};

// error plumbing
void set_error(const std::string& s);
// pg_rve_desc -> RveSpec with the argument checks of the mesh builders (pg_capi.cu)
int rve_spec_from_desc(const pg_rve_desc* rve, RveSpec& spec, const char* who);
// IGFEM preprocessing and sparsity on the GPU, the same HostMesh as build_mesh (pg_mesh_gpu.cu)
int build_mesh_device(const RveSpec& spec, int device, HostMesh& out);
// device context of a host mesh (pg_capi.cu)
int ctx_create(HostMesh hm, int device, Ctx& c);  // the context keeps the mesh (move it in)
int ensure_tri_map(Ctx& c);  // the row-tile kernel's block maps, built on first use
void free_ctx(Ctx& c);
int cuda_fail(cudaError_t e, const char* where);

// assembly entry points (pg_assemble.cu)
void upload_tables();
int launch_assemble(Ctx& c, const double* U, double dt, bool want_f, bool want_K, cudaStream_t s);
int launch_to_fp32(Ctx& c, cudaStream_t s);
// Problem::compute_stress_strain at every volumetric point into c.qp_out (7 per point) and,
// with mean7, the J W-weighted means of strain and stress and the total J W
int stress_strain(Ctx& c, const double* U, cudaStream_t s, double* mean7);
// point offsets per element and the recovery's tables (first call builds them)
int stress_prepare(Ctx& c);
// the reference's legacy ASCII VTK file and cohesive openings CSV of the context's state
int write_vtk(Ctx& c, const std::string& path, double t);
int write_cohesive_openings(Ctx& c, const std::string& path);
int autotune_assembly(Ctx& c, int reps, float* ms_tri, float* ms_cut);
// shape sensitivity (pg_sens.cu): per-node inclusion / velocity and the cut-kernel passes
// Arguments of the cut elements' shape-sensitivity kernel (pg_assemble.cu)
struct CutArgs {
    int n_cut;                      // elements of this launch (one size class)
    int first;                      // its first element in the class-ordered arrays
    const int* __restrict__ cut_nodes;
    const int* __restrict__ cut_tmpl;
    const int* __restrict__ cut_child_mat;
    const int* __restrict__ cut_coh_qp0;
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ u;
    const double* __restrict__ dmat;
    const double* __restrict__ isv_c;
    DevCohLaw coh;
    double dt;
    // the element's enrichment nodes of its `which`-th inclusion move by
    // sgn * h_rel * r * velocity, and the element's internal force dotted
    // with wsens goes to sens[inclusion]
    const int* node_inc;
    const double* vel;
    const double* wsens;
    const double* radius;
    double* sens;
    double h_rel, sgn;
    int which;
    // analytic passes: parameter slot of (inclusion, kind) at param_of[3 inclusion + kind]
    // (-1: not a parameter); vel is the velocity field of this pass's kind
    const int* param_of;
    int kind;
};
CutArgs cut_args(const Ctx& c, const double* U, double dt);
void launch_cut_sens_ad(const Ctx& c, const CutArgs& ca, cudaStream_t s);
// fold order of the cut elements' deterministic assembly, built on the GPU
// from the context's class-ordered cut tables (pg_mesh_gpu.cu)
int build_fold_device(Ctx& c, const std::vector<uint8_t>& node_enr, int n_entries);
int device_point_count(int tmpl);  // quadrature points of a cut template on the device
constexpr int kCutPointInts = 16;  // ints per point record of the cut-row kernel
void build_cut_points(const std::vector<int>& nodes, const std::vector<int>& tmpl, const std::vector<int>& chm,
                      const std::vector<long long>& roff, const int* class_off, std::vector<int>& out,
                      std::vector<int>& pt_off);
// per size class and CTA size (2, 4, 8 warps): the widest span of rows
// (doubles) of the elements one CTA of k_cut_elems takes
void cut_row_spans(const std::vector<long long>& roff, const int* class_off, int span[4][3]);
constexpr int kCutCtaWarps[3] = {2, 4, 8};
// elements of size class NL per CTA of k_cut_elems: one thread per local function
__host__ __device__ constexpr int cut_elems_per_cta(int threads, int nl) { return threads / nl; }
void launch_cut_sens(const Ctx& c, const CutArgs& ca, cudaStream_t s);

// solver entry points (pg_solve.cu)
int solve_linear_system(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s);
// mask(K) x = b for x (x starts at 0); b = c.b (masked); result in c.dx
int krylov_solve(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s);
// out = mask(b - K x) (b nullable: 0); returns ||out||^2
double residual_into(Ctx& c, cudaStream_t s, const double* x, const double* b, double* out);
// geometric multigrid (pg_mg.cu)
int mg_pcg_solve(Ctx& c, const pg_solver_cfg& cfg, pg_solve_stats& st, cudaStream_t s);
int mg_prepare(Ctx& c, bool f32, bool modes, cudaStream_t s);
void mg_precondition(Ctx& c, bool f32, cudaStream_t s, const double* r, double* z);
void mg_free(Ctx& c);
// ||v||^2 of a device vector (synchronises)
double dev_norm2(Ctx& c, const double* v, int n, cudaStream_t s);
void set_prescribed(Ctx& c, double t_frac, cudaStream_t s);

// learned predictor (pg_predict.cu)
int launch_features(Ctx& c, const pg_pred_history& h, float* X, cudaStream_t s);
// U (free DOFs) = linear extrapolation + g * curvature term, g = scale * the curvature-weighted
// mean of (1 + Y) (Y null: g = 0, the linear extrapolation); g_used (nullable) receives g
int launch_apply(Ctx& c, const pg_pred_history& h, const float* Y, double scale, double* U, cudaStream_t s,
                 double* g_used = nullptr);
double predictor_app(const Ctx& c);
double predictor_residual(Ctx& c, const double* U, double dt, cudaStream_t s);

// Newton (pg_newton.cu)
// r_base > 0: rtol is relative to it instead of the predictor's residual
int newton_load_step(Ctx& c, double t_frac, double dt, const pg_newton_cfg& cfg, pg_step_stats& st, cudaStream_t s,
                     double r_base = 0.0);

}  // namespace pgb

struct pg_ctx {
    pgb::Ctx c;
};

#define PG_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) return ::pgb::cuda_fail(_e, #call);         \
    } while (0)
