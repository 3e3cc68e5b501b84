// extern "C" entry points of libpigfem_b200 (declared in include/pigfem_b200.h).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "pg_internal.cuh"
#include "pg_solve_kernels.cuh"

namespace pgb {

namespace {
thread_local std::string g_last_error;

template <typename T>
int dev_upload(T** dst, const std::vector<T>& src) {
    *dst = nullptr;
    if (src.empty()) return PG_OK;
    PG_CUDA(cudaMalloc((void**)dst, src.size() * sizeof(T)));
    PG_CUDA(h2d_sync(*dst, src.data(), src.size() * sizeof(T)));
    return PG_OK;
}

template <typename T>
int dev_alloc(T** dst, size_t n) {
    *dst = nullptr;
    if (n == 0) n = 1;
    PG_CUDA(cudaMalloc((void**)dst, n * sizeof(T)));
    PG_CUDA(fill_sync(*dst, 0, n * sizeof(T)));
    return PG_OK;
}


// D = E/((1+nu)(1-2nu)) [[1-nu, nu, 0], [nu, 1-nu, 0], [0, 0, (1-2nu)/2]]
// (material_lei.cpp:62-77; plane stress :78-84)
void dmat_coeffs(const Material& m, bool plane_strain, double out[3]) {
    if (plane_strain) {
        const double coef = m.E / ((1.0 + m.nu) * (1.0 - 2.0 * m.nu));
        out[0] = coef * (1.0 - m.nu);
        out[1] = coef * (m.nu);
        out[2] = coef * (1.0 - 2.0 * m.nu) / 2.0;
    } else {
        const double coef = m.E / (1.0 - m.nu * m.nu);
        out[0] = coef;
        out[1] = coef * (m.nu);
        out[2] = coef * (1.0 - m.nu) / 2.0;
    }
}

cudaStream_t pick(Ctx& c, void* s) { return s ? (cudaStream_t)s : c.stream; }

}  // namespace

void free_ctx(Ctx& c) {
    mg_free(c);
    void* ptrs[] = {c.xi, c.mw, c.nq_ptr, c.nq_list, c.featX, c.featY, c.b, c.res, c.Ut, c.Uprev, c.Uold, c.Uold2, c.isv_prev, c.red_ws, c.V, c.hbuf, c.x, c.y, c.elem4, c.row_ptr, c.col, c.diag, c.ne_ptr, c.ne_list, c.tri_map[0], c.tri_map[1], c.grid_emat, c.dmat, c.cut_nodes, c.cut_tmpl,
                    c.cut_child_mat, c.cut_coh_qp0, c.cut_slot_ptr, c.cut_slot, c.cut_rows, c.cut_row_off, c.cut_pts,
                    c.cut_pt_off, c.cut_kdir, c.fold_Km_slot, c.fold_Km_rng,
                    c.grid_rves, c.grid_tiles[0], c.grid_tiles[1], c.qp_off, c.qp_elem_cut, c.qp_cut_elem,
                    c.qp_class_off, c.qp_out,
                    c.cut_ke, c.cut_fe, c.cut_kpos, c.cut_fpos, c.fold_K_slot, c.fold_K_ptr, c.fold_f_node,
                    c.fold_f_ptr, c.coh_rec, c.coh_rows, c.K, c.Kf, c.fixed, c.ubar,
                    c.U, c.F, c.isv_c, c.isv_t, c.r, c.z, c.p, c.q, c.dx, c.minv, c.rf, c.zf, c.pf, c.qf, c.xf,
                    c.minvf, c.scal, c.iflags};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (c.h_scal) cudaFreeHost(c.h_scal);
    if (c.h_iflags) cudaFreeHost(c.h_iflags);
    if (c.ev0) cudaEventDestroy(c.ev0);
    if (c.ev1) cudaEventDestroy(c.ev1);
    for (cudaEvent_t e : {c.ea0, c.ea1, c.ea2, c.fork_ev, c.join_ev})
        if (e) cudaEventDestroy(e);
    if (c.aux) cudaStreamDestroy(c.aux);
    if (c.stream) cudaStreamDestroy(c.stream);
}

void set_error(const std::string& s) { g_last_error = s; }

int ensure_tri_map(Ctx& c) {
    for (int v = 0; v < kTriTileVariants; ++v) {
        if (c.tri_map[v]) continue;
        std::vector<int> tm;
        build_tri_map(c.hm, kTriTileSizes[v], tm);
        const int rc = dev_upload(&c.tri_map[v], tm);
        if (rc) return rc;
    }
    return PG_OK;
}

int cuda_fail(cudaError_t e, const char* where) {
    g_last_error = std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e);
    return PG_ERR_CUDA;
}

int ctx_create(HostMesh mesh, int device, Ctx& c) {
    c.device = device;
    PG_CUDA(cudaSetDevice(device));
    upload_tables();
    PG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    PG_CUDA(cudaStreamCreateWithFlags(&c.aux, cudaStreamNonBlocking));
    PG_CUDA(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
    PG_CUDA(cudaEventCreateWithFlags(&c.join_ev, cudaEventDisableTiming));
    PG_CUDA(cudaEventCreate(&c.ev0));
    PG_CUDA(cudaEventCreate(&c.ev1));
    PG_CUDA(cudaEventCreate(&c.ea0));
    PG_CUDA(cudaEventCreate(&c.ea1));
    PG_CUDA(cudaEventCreate(&c.ea2));
    c.hm = std::move(mesh);
    const HostMesh& hm = c.hm;
    c.n_nodes = hm.n_nodes();
    c.n_reg = hm.n_reg;
    c.n_elem = hm.n_elem;
    c.n_cut = hm.n_cut;
    c.n_blocks = hm.n_blocks();
    c.n_dof = hm.n_dof();
    c.n_coh_qp = hm.n_coh_qp;
    c.coh.law = hm.spec.coh.law;
    for (int k = 0; k < 5; ++k) c.coh.p[k] = hm.spec.coh.p[k];

    auto now = [] { return std::chrono::steady_clock::now(); };
    auto secs = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    auto t_phase = now();
    int rc;
    if ((rc = dev_upload(&c.x, hm.x))) return rc;
    if ((rc = dev_upload(&c.y, hm.y))) return rc;
    std::vector<int4> e4(hm.n_elem);
    parallel_for(hm.n_elem, 1 << 16, [&](long long e) {
        e4[e] = make_int4(hm.conn[3 * e], hm.conn[3 * e + 1], hm.conn[3 * e + 2], hm.elem_mat[e]);
    });
    if ((rc = dev_upload(&c.elem4, e4))) return rc;
    if ((rc = dev_upload(&c.row_ptr, hm.row_ptr))) return rc;
    if ((rc = dev_upload(&c.col, hm.col))) return rc;
    if ((rc = dev_upload(&c.diag, hm.diag_slot))) return rc;
    if ((rc = dev_upload(&c.ne_ptr, hm.ne_ptr))) return rc;
    if ((rc = dev_upload(&c.ne_list, hm.ne_list))) return rc;
    c.setup_s[0] = secs(t_phase, now());
    t_phase = now();
    // (the row-tile kernel's block maps are built on its first use: ensure_tri_map)
    long long grid_elems = 0;
    for (const auto& gb : hm.grids) grid_elems += 2LL * gb.nx * gb.ny;
    if (!hm.grids.empty() && grid_elems == hm.n_elem && grid_pattern_ok(hm)) {
        // structured background grids (one per RVE of a batch): the grid kernel
        // applies, through a tile table per tile height over all of them
        std::vector<int> em(hm.n_elem);
        parallel_for(hm.n_elem, 1 << 16, [&](long long e) { em[e] = hm.elem_cut[e] >= 0 ? -1 : hm.elem_mat[e]; });
        if ((rc = dev_upload(&c.grid_emat, em))) return rc;
        std::vector<int4> rves;
        for (const auto& gb : hm.grids) rves.push_back(make_int4(gb.nx, gb.ny, gb.node_off, gb.elem_off));
        if ((rc = dev_upload(&c.grid_rves, rves))) return rc;
        for (int h = 0; h < 2; ++h) {
            const int tr = h == 0 ? 2 : 4;
            std::vector<int4> tiles;
            for (int r = 0; r < (int)hm.grids.size(); ++r) {
                const auto& gb = hm.grids[r];
                for (int J0 = 0; J0 <= gb.ny; J0 += tr)
                    for (int I0 = 0; I0 <= gb.nx; I0 += kGridTileCols) tiles.push_back(make_int4(r, I0, J0, 0));
            }
            c.n_grid_tiles[h] = (int)tiles.size();
            if ((rc = dev_upload(&c.grid_tiles[h], tiles))) return rc;
        }
    } else {
        c.tuning.tri_grid = 0;
    }
    // enrichment nodes: those beyond the regular nodes of their grid block (a
    // mesh without blocks: beyond n_reg)
    std::vector<uint8_t> node_enr(hm.n_nodes(), 0);
    if (hm.grids.empty()) {
        for (int n = hm.n_reg; n < hm.n_nodes(); ++n) node_enr[n] = 1;
    } else {
        for (size_t r = 0; r < hm.grids.size(); ++r) {
            const int end = r + 1 < hm.grids.size() ? hm.grids[r + 1].node_off : hm.n_nodes();
            for (int n = hm.grids[r].node_off + hm.grids[r].n_reg; n < end; ++n) node_enr[n] = 1;
        }
    }
    c.setup_s[1] = secs(t_phase, now());
    t_phase = now();
    std::vector<double> dm(3 * hm.spec.materials.size());
    for (size_t m = 0; m < hm.spec.materials.size(); ++m) dmat_coeffs(hm.spec.materials[m], hm.spec.plane_strain, &dm[3 * m]);
    if ((rc = dev_upload(&c.dmat, dm))) return rc;
    if (hm.n_cut > 0) {
        // cut elements grouped by size class (each class in mesh order); every
        // per-element array below is stored in that order, with the element's
        // local nodes (3 parents, then enrichment slots) as one flat list
        std::vector<int> order;
        order.reserve(hm.n_cut);
        for (int k = 0; k < kCutClasses; ++k) {
            c.cut_class_off[k] = (int)order.size();
            const int lo = k == 0 ? 0 : kCutClassNl[k - 1];
            for (int ci = 0; ci < hm.n_cut; ++ci) {
                const int nl = 3 + cut_template(hm.cut_tmpl[ci]).n_enr;
                if (nl > lo && nl <= kCutClassNl[k]) order.push_back(ci);
            }
        }
        c.cut_class_off[kCutClasses] = (int)order.size();
        if (order.size() != (size_t)hm.n_cut) {
            set_error("cut element with more local nodes than the largest size class");
            return PG_ERR_MESH;
        }
        const int nc = hm.n_cut;
        constexpr int S = kMaxElemNodes;
        std::vector<int> nodes((size_t)kCutNodeStride * nc, -1), tmpl(nc), chm((size_t)kMaxChildren * nc), qp0(nc);
        std::vector<int> sp(nc + 1, 0), sl;
        for (int oi = 0; oi < nc; ++oi) {
            const int nl = 3 + cut_template(hm.cut_tmpl[order[oi]]).n_enr;
            sp[oi + 1] = sp[oi] + nl * nl;
        }
        sl.resize(sp[nc]);
        // every element fills its own ranges: in parallel
        parallel_for(nc, 4096, [&](long long oi) {
            const int ci = order[oi], e = hm.cut_elem[ci];
            const int nl = 3 + cut_template(hm.cut_tmpl[ci]).n_enr;
            for (int v = 0; v < 3; ++v) nodes[(size_t)kCutNodeStride * oi + v] = hm.conn[3 * e + v];
            for (int k = 0; k < nl - 3; ++k) nodes[(size_t)kCutNodeStride * oi + 3 + k] = hm.cut_enr[(size_t)ci * kMaxEnr + k];
            tmpl[oi] = hm.cut_tmpl[ci];
            for (int k = 0; k < kMaxChildren; ++k) chm[(size_t)kMaxChildren * oi + k] = hm.cut_child_mat[(size_t)ci * kMaxChildren + k];
            qp0[oi] = hm.cut_coh_qp0[ci];
            int* dst = &sl[sp[oi]];
            for (int a = 0; a < nl; ++a)
                for (int b = 0; b < nl; ++b) *dst++ = hm.cut_slot[(size_t)ci * S * S + a * S + b];
        });
        if ((rc = dev_upload(&c.cut_nodes, nodes))) return rc;
        if ((rc = dev_upload(&c.cut_tmpl, tmpl))) return rc;
        if ((rc = dev_upload(&c.cut_child_mat, chm))) return rc;
        if ((rc = dev_upload(&c.cut_coh_qp0, qp0))) return rc;
        if ((rc = dev_upload(&c.cut_slot_ptr, sp))) return rc;
        if ((rc = dev_upload(&c.cut_slot, sl))) return rc;
        // where each cut element's quadrature rows go (4 + 2 NL doubles per point, point-major)
        std::vector<long long> roff(nc + 1, 0);
        for (int k = 0; k < kCutClasses; ++k)
            for (int oi = c.cut_class_off[k]; oi < c.cut_class_off[k + 1]; ++oi)
                roff[oi + 1] = roff[oi] + (long long)device_point_count(tmpl[oi]) * (4 + 2 * kCutClassNl[k]);
        std::vector<int> pts, pt_off;
        build_cut_points(nodes, tmpl, chm, roff, c.cut_class_off, pts, pt_off);
        c.n_cut_pts = (int)(pts.size() / kCutPointInts) - 1;  // the last record is the sentinel
        cut_row_spans(roff, c.cut_class_off, c.cut_span);
        if ((rc = dev_upload(&c.cut_row_off, roff)) || (rc = dev_upload(&c.cut_pts, pts)) ||
            (rc = dev_upload(&c.cut_pt_off, pt_off)))
            return rc;
        c.cut_rows_len = roff[nc];  // allocated by the stress recovery, the only user of rows in global memory
        // cohesive Gauss points: the owning element, sub-element and point
        if (hm.n_coh_qp > 0) {
            std::vector<int> rec(hm.n_coh_qp, -1);
            for (int oi = 0; oi < nc; ++oi) {
                const CutTemplate& T = cut_template(tmpl[oi]);
                for (int ce = 0; ce < T.n_coh; ++ce)
                    for (int q = 0; q < 2; ++q) rec[qp0[oi] + 2 * ce + q] = (oi << 8) | (ce << 1) | q;
            }
            for (int v : rec)
                if (v < 0) {
                    set_error("cohesive Gauss point not owned by any cut element");
                    return PG_ERR_MESH;
                }
            if ((rc = dev_upload(&c.coh_rec, rec)) ||
                (rc = dev_alloc(&c.coh_rows, (size_t)kCohRowDoubles * hm.n_coh_qp)))
                return rc;
        }
        c.setup_s[2] = secs(t_phase, now());
        t_phase = now();
        // deterministic assembly: the pair buffers and the fold order (built on the GPU)
        if ((rc = dev_alloc(&c.cut_ke, 4 * std::max<size_t>(1, sl.size()))) ||
            (rc = dev_alloc(&c.cut_fe, 2 * std::max<size_t>(1, sl.size()))))
            return rc;
        if ((rc = build_fold_device(c, node_enr, (int)sl.size()))) return rc;
        c.setup_s[3] = secs(t_phase, now());
    }
    const size_t nb = (size_t)c.n_blocks, nd = (size_t)c.n_dof, nn = (size_t)c.n_nodes;
    if ((rc = dev_alloc(&c.K, 4 * nb))) return rc;
    if ((rc = dev_alloc(&c.Kf, 4 * nb))) return rc;
    if ((rc = dev_upload(&c.fixed, hm.fixed))) return rc;
    if ((rc = dev_upload(&c.ubar, hm.ubar))) return rc;
    if ((rc = dev_alloc(&c.U, nd))) return rc;
    if ((rc = dev_alloc(&c.F, nd))) return rc;
    if ((rc = dev_alloc(&c.isv_c, (size_t)std::max(1, hm.n_coh_qp)))) return rc;
    if ((rc = dev_alloc(&c.isv_t, (size_t)std::max(1, hm.n_coh_qp)))) return rc;
    if ((rc = dev_alloc(&c.isv_prev, (size_t)std::max(1, hm.n_coh_qp)))) return rc;
    for (double** v : {&c.r, &c.z, &c.p, &c.q, &c.dx, &c.b, &c.res, &c.Ut, &c.Uprev, &c.Uold, &c.Uold2, &c.xi})
        if ((rc = dev_alloc(v, nd))) return rc;
    if ((rc = dev_alloc(&c.minv, 4 * nn))) return rc;
    if ((rc = dev_alloc(&c.mw, 2 * nd))) return rc;
    for (float** v : {&c.rf, &c.zf, &c.pf, &c.qf, &c.xf})
        if ((rc = dev_alloc(v, nd))) return rc;
    if ((rc = dev_alloc(&c.minvf, 4 * nn))) return rc;
    if ((rc = dev_alloc(&c.hbuf, 128))) return rc;
    if ((rc = dev_alloc(&c.scal, 64))) return rc;
    {
        // the largest grid of a reduction: a thread per DOF, or kRowLanes per node row
        const int cap = (int)std::max<long long>({((long long)nd + kThreads - 1) / kThreads,
                                                  ((long long)kRowLanes * (long long)nn + kThreads - 1) / kThreads,
                                                  1184LL}) + 1;
        if ((rc = dev_alloc(&c.red_ws, red_ws_doubles(cap)))) return rc;
        const double capd = (double)cap;
        PG_CUDA(h2d_sync(c.red_ws, &capd, sizeof(double)));
        c.red_active = c.red_ws;
    }
    if ((rc = dev_alloc(&c.iflags, 64))) return rc;
    PG_CUDA(cudaMallocHost((void**)&c.h_scal, 64 * sizeof(double)));
    PG_CUDA(cudaMallocHost((void**)&c.h_iflags, 64 * sizeof(int)));
    // prescribed values at load factor 1
    set_prescribed(c, 1.0, c.stream);
    PG_CUDA(cudaStreamSynchronize(c.stream));
    return PG_OK;
}

}  // namespace pgb

namespace pgb {
const char* last_error_cstr() { return g_last_error.c_str(); }
}  // namespace pgb

using namespace pgb;

#define PG_GUARD_CTX(c)                                   \
    do {                                                  \
        if (!(c)) { set_error("null context"); return PG_ERR_ARG; } \
        cudaSetDevice((c)->c.device);                     \
    } while (0)

namespace pgb {

// pg_rve_desc -> RveSpec with the argument checks both mesh builders share
int rve_spec_from_desc(const pg_rve_desc* rve, RveSpec& spec, const char* who) {
    const std::string w(who);
    spec.nx = rve->nx;
    spec.ny = rve->ny;
    spec.x0 = rve->x0;
    spec.x1 = rve->x1;
    spec.y0 = rve->y0;
    spec.y1 = rve->y1;
    if (rve->n_materials <= 0 || !rve->mat_E || !rve->mat_nu) { set_error(w + ": no materials"); return PG_ERR_ARG; }
    for (int m = 0; m < rve->n_materials; ++m) spec.materials.push_back({rve->mat_E[m], rve->mat_nu[m]});
    spec.matrix_mat = rve->matrix_mat;
    if (rve->n_inclusions < 0 || (rve->n_inclusions > 0 && (!rve->inc_cx || !rve->inc_cy || !rve->inc_r || !rve->inc_mat))) {
        set_error(w + ": inclusion arrays missing");
        return PG_ERR_ARG;
    }
    for (int i = 0; i < rve->n_inclusions; ++i)
        spec.inclusions.push_back({rve->inc_cx[i], rve->inc_cy[i], rve->inc_r[i], rve->inc_mat[i]});
    spec.plane_strain = rve->plane_strain != 0;
    spec.cohesive = rve->cohesive != 0;
    spec.coh.law = rve->coh_law;
    for (int k = 0; k < 5; ++k) spec.coh.p[k] = rve->coh_params[k];
    if (spec.cohesive && spec.coh.law == PG_COH_BILINEAR && !(spec.coh.p[4] >= 0.0)) {
        set_error(w + ": the bilinear law's viscosity must be >= 0");
        return PG_ERR_ARG;
    }
    if (spec.cohesive && spec.coh.law != PG_COH_OP && spec.coh.law != PG_COH_BILINEAR) {
        set_error(w + ": unknown cohesive law");
        return PG_ERR_ARG;
    }
    spec.strain = rve->strain;
    return PG_OK;
}

}  // namespace pgb

extern "C" {

const char* pg_last_error(void) { return last_error_cstr(); }
const char* pg_version(void) { return "pigfem_b200 0.1 (sm_100a)"; }

int pg_mesh_build(const pg_rve_desc* rve, pg_mesh** out) {
    if (!rve || !out) { set_error("pg_mesh_build: null argument"); return PG_ERR_ARG; }
    *out = nullptr;
    RveSpec spec;
    int rc = rve_spec_from_desc(rve, spec, "pg_mesh_build");
    if (rc != PG_OK) return rc;
    pg_mesh* m = new (std::nothrow) pg_mesh;
    if (!m) { set_error("pg_mesh_build: out of host memory"); return PG_ERR_ARG; }
    std::string err;
    try {
        err = build_mesh(spec, m->m);
    } catch (const std::exception& ex) {
        err = std::string("host exception: ") + ex.what();
    }
    if (!err.empty()) {
        delete m;
        set_error("pg_mesh_build: " + err);
        return PG_ERR_MESH;
    }
    *out = m;
    return PG_OK;
}

int pg_mesh_build_device(const pg_rve_desc* rve, int32_t device, pg_mesh** out) {
    if (!rve || !out) { set_error("pg_mesh_build_device: null argument"); return PG_ERR_ARG; }
    *out = nullptr;
    RveSpec spec;
    int rc = rve_spec_from_desc(rve, spec, "pg_mesh_build_device");
    if (rc != PG_OK) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("pg_mesh_build_device: no CUDA device (this library has no CPU fallback)");
        return PG_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) { set_error("pg_mesh_build_device: invalid device"); return PG_ERR_ARG; }
    pg_mesh* m = new (std::nothrow) pg_mesh;
    if (!m) { set_error("pg_mesh_build_device: out of host memory"); return PG_ERR_ARG; }
    try {
        rc = build_mesh_device(spec, device, m->m);
    } catch (const std::exception& ex) {
        set_error(std::string("pg_mesh_build_device: host exception: ") + ex.what());
        rc = PG_ERR_MESH;
    }
    if (rc != PG_OK) {
        delete m;
        return rc;
    }
    *out = m;
    return PG_OK;
}

int pg_mesh_info_get(const pg_mesh* mm, pg_mesh_info* info) {
    if (!mm || !info) { set_error("pg_mesh_info_get: null argument"); return PG_ERR_ARG; }
    const HostMesh& m = mm->m;
    info->n_nodes = m.n_nodes();
    info->n_regular_nodes = m.n_reg;
    info->n_enrichment_nodes = m.n_enr;
    info->n_elements = m.n_elem;
    info->n_cut_elements = m.n_cut;
    info->n_cohesive_qp = m.n_coh_qp;
    info->n_dof = m.n_dof();
    info->n_free_dof = m.n_free;
    info->n_blocks = m.n_blocks();
    info->n_moved_nodes = m.n_moved;
    return PG_OK;
}

int pg_mesh_export(const pg_mesh* mm, double* xy, int32_t* conn, int32_t* elem_mat, int32_t* elem_cut, int32_t* ref_dof,
                   uint8_t* fixed, double* ubar) {
    if (!mm) { set_error("pg_mesh_export: null mesh"); return PG_ERR_ARG; }
    const HostMesh& m = mm->m;
    if (xy)
        for (int n = 0; n < m.n_nodes(); ++n) { xy[2 * n] = m.x[n]; xy[2 * n + 1] = m.y[n]; }
    if (conn) std::memcpy(conn, m.conn.data(), m.conn.size() * sizeof(int));
    if (elem_mat) std::memcpy(elem_mat, m.elem_mat.data(), m.elem_mat.size() * sizeof(int));
    if (elem_cut) std::memcpy(elem_cut, m.elem_cut.data(), m.elem_cut.size() * sizeof(int));
    if (ref_dof) std::memcpy(ref_dof, m.ref_dof.data(), m.ref_dof.size() * sizeof(int));
    if (fixed) std::memcpy(fixed, m.fixed.data(), m.fixed.size());
    if (ubar) std::memcpy(ubar, m.ubar.data(), m.ubar.size() * sizeof(double));
    return PG_OK;
}

int pg_mesh_export_cut(const pg_mesh* mm, int32_t* cut_elem, int32_t* cut_tmpl, int32_t* cut_enr, int32_t* cut_child_mat,
                       int32_t* cut_coh_qp0) {
    if (!mm) { set_error("pg_mesh_export_cut: null mesh"); return PG_ERR_ARG; }
    const HostMesh& m = mm->m;
    if (cut_elem && m.n_cut) std::memcpy(cut_elem, m.cut_elem.data(), m.n_cut * sizeof(int));
    if (cut_tmpl && m.n_cut) std::memcpy(cut_tmpl, m.cut_tmpl.data(), m.n_cut * sizeof(int));
    if (cut_enr && m.n_cut) std::memcpy(cut_enr, m.cut_enr.data(), m.cut_enr.size() * sizeof(int));
    if (cut_child_mat && m.n_cut) std::memcpy(cut_child_mat, m.cut_child_mat.data(), m.cut_child_mat.size() * sizeof(int));
    if (cut_coh_qp0 && m.n_cut) std::memcpy(cut_coh_qp0, m.cut_coh_qp0.data(), m.n_cut * sizeof(int));
    return PG_OK;
}

int pg_mesh_export_pattern(const pg_mesh* mm, int32_t* row_ptr, int32_t* col) {
    if (!mm) { set_error("pg_mesh_export_pattern: null mesh"); return PG_ERR_ARG; }
    const HostMesh& m = mm->m;
    if (row_ptr) std::memcpy(row_ptr, m.row_ptr.data(), m.row_ptr.size() * sizeof(int));
    if (col) std::memcpy(col, m.col.data(), m.col.size() * sizeof(int));
    return PG_OK;
}

// 80 int32 per template: n_cut_edges, n_enr, n_child, n_coh, cut_edge[6],
// enr_inc_node[6], child_n[4], child_mat_node[4], child_nodes[4][6], coh_nodes[3][4],
// then padding to 80.
int pg_template_table(int32_t* out, int32_t* n) {
    const int nt = n_cut_templates();
    if (n) *n = nt;
    if (!out) return PG_OK;
    for (int t = 0; t < nt; ++t) {
        const CutTemplate& T = cut_template(t);
        int32_t* o = out + 80 * t;
        std::memset(o, 0xff, 80 * sizeof(int32_t));
        o[0] = T.n_cut_edges; o[1] = T.n_enr; o[2] = T.n_child; o[3] = T.n_coh;
        for (int i = 0; i < 6; ++i) { o[4 + i] = i < T.n_cut_edges ? T.cut_edge[i] : -1; o[10 + i] = i < T.n_cut_edges ? T.enr_inc_node[i] : -1; }
        for (int c = 0; c < 4; ++c) {
            o[16 + c] = c < T.n_child ? T.child_n[c] : 0;
            o[20 + c] = c < T.n_child ? T.child_mat_node[c] : -2;
            for (int k = 0; k < 6; ++k) o[24 + 6 * c + k] = (c < T.n_child && k < T.child_n[c]) ? T.child_nodes[c][k] : -1;
        }
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 4; ++k) o[48 + 4 * c + k] = c < T.n_coh ? T.coh_nodes[c][k] : -1;
    }
    return PG_OK;
}

void pg_mesh_destroy(pg_mesh* m) { delete m; }

int pg_ctx_create(const pg_mesh* m, int32_t device, pg_ctx** out) {
    if (!m || !out) { set_error("pg_ctx_create: null argument"); return PG_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("pg_ctx_create: no CUDA device (this library has no CPU fallback)");
        return PG_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) { set_error("pg_ctx_create: invalid device"); return PG_ERR_ARG; }
    pg_ctx* c = new (std::nothrow) pg_ctx;
    if (!c) { set_error("pg_ctx_create: out of host memory"); return PG_ERR_ARG; }
    const int rc = ctx_create(m->m, device, c->c);
    if (rc != PG_OK) {
        free_ctx(c->c);
        delete c;
        return rc;
    }
    *out = c;
    return PG_OK;
}

void pg_ctx_destroy(pg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->c.device);
    free_ctx(c->c);
    delete c;
}

int pg_ctx_autotune(pg_ctx* c, int32_t reps, float* ms_tri, float* ms_cut) {
    PG_GUARD_CTX(c);
    cudaSetDevice(c->c.device);
    return autotune_assembly(c->c, reps, ms_tri, ms_cut);
}

int pg_ctx_tuning(pg_ctx* c, int32_t* tri_tile_nodes, int32_t* tri_persistent, int32_t* cut_warps) {
    PG_GUARD_CTX(c);
    if (tri_tile_nodes)
        *tri_tile_nodes = c->c.tuning.tri_grid ? c->c.tuning.grid_block : kTriTileSizes[c->c.tuning.tri_variant];
    if (tri_persistent) *tri_persistent = c->c.tuning.tri_persistent;
    if (cut_warps) *cut_warps = c->c.tuning.cut_warps;
    return PG_OK;
}

int pg_ctx_set_tuning(pg_ctx* c, int32_t tri_tile_nodes, int32_t tri_persistent, int32_t cut_warps) {
    PG_GUARD_CTX(c);
    int v = -1;
    for (int k = 0; k < kTriTileVariants; ++k)
        if (kTriTileSizes[k] == tri_tile_nodes) v = k;
    const bool grid = tri_tile_nodes == 128 || tri_tile_nodes == 256;
    if ((v < 0 && !(grid && c->c.grid_emat)) || (tri_persistent != 0 && tri_persistent != 1) ||
        (cut_warps != 2 && cut_warps != 4 && cut_warps != 8)) {
        set_error("pg_ctx_set_tuning: tile 32 or 64 (row tiles), 128 or 256 (threads per CTA of the structured-grid "
                  "kernel, meshes with one grid), persistent 0 or 1, warps 2, 4 or 8");
        return PG_ERR_ARG;
    }
    c->c.tuning.tri_grid = grid ? 1 : 0;
    if (grid) c->c.tuning.grid_block = tri_tile_nodes;
    if (!grid) c->c.tuning.tri_variant = v;
    c->c.tuning.tri_persistent = tri_persistent;
    c->c.tuning.cut_warps = cut_warps;
    return PG_OK;
}

int pg_ctx_cut_overlap(pg_ctx* c, int32_t set, int32_t* get) {
    PG_GUARD_CTX(c);
    if (set >= 0) {
        if (set > 2) { set_error("pg_ctx_cut_overlap: 0 (after the grid kernel), 1 or 2 (beside it)"); return PG_ERR_ARG; }
        c->c.tuning.cut_overlap = set;
    }
    if (get) *get = c->c.tuning.cut_overlap;
    return PG_OK;
}

int pg_ctx_sync(pg_ctx* c) {
    PG_GUARD_CTX(c);
    PG_CUDA(cudaStreamSynchronize(c->c.stream));
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int pg_assemble_linear(pg_ctx* c, void* stream) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    const int rc = launch_assemble(x, x.U, 0.0, false, true, pick(x, stream));
    if (rc == PG_OK) x.assembled = true;
    return rc;
}

int pg_assemble_linear_host(pg_ctx* c, const double* xy_host, double* k_host) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    cudaStream_t s = x.stream;
    if (xy_host) {
        // de-interleave on the device from a staging copy in the F work vector
        PG_CUDA(cudaMemcpyAsync(x.F, xy_host, 2 * (size_t)x.n_nodes * sizeof(double), cudaMemcpyHostToDevice, s));
        PG_CUDA(cudaMemcpy2DAsync(x.x, sizeof(double), x.F, 2 * sizeof(double), sizeof(double), x.n_nodes,
                                  cudaMemcpyDeviceToDevice, s));
        PG_CUDA(cudaMemcpy2DAsync(x.y, sizeof(double), x.F + 1, 2 * sizeof(double), sizeof(double), x.n_nodes,
                                  cudaMemcpyDeviceToDevice, s));
    }
    int rc = launch_assemble(x, x.U, 0.0, false, true, s);
    if (rc != PG_OK) return rc;
    x.assembled = true;
    if (k_host) PG_CUDA(cudaMemcpyAsync(k_host, x.K, 4 * (size_t)x.n_blocks * sizeof(double), cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    return PG_OK;
}

int pg_assemble_nonlinear(pg_ctx* c, const double* U_dev, double dt, int32_t want_f, int32_t want_K, void* stream) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!want_f && !want_K) return PG_OK;
    cudaStream_t s = pick(x, stream);
    const double* U = U_dev ? U_dev : x.U;
    if (want_f) PG_CUDA(cudaMemsetAsync(x.F, 0, (size_t)x.n_dof * sizeof(double), s));
    const int rc = launch_assemble(x, U, dt, want_f != 0, want_K != 0, s);
    if (rc == PG_OK && want_K) x.assembled = true;
    return rc;
}

int pg_stress_strain(pg_ctx* c, const double* U_dev, double* points_host, int64_t* n_points, int32_t* elem_point_off,
                     double* mean) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    int rc = stress_prepare(x);
    if (rc != PG_OK) return rc;
    if (n_points) *n_points = x.n_qp_total;
    if (elem_point_off)
        PG_CUDA(cudaMemcpy(elem_point_off, x.qp_off, ((size_t)x.n_elem + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    if (!points_host && !mean) return PG_OK;
    cudaStream_t s = x.stream;
    rc = stress_strain(x, U_dev ? U_dev : x.U, s, mean);
    if (rc != PG_OK) return rc;
    if (points_host)
        PG_CUDA(cudaMemcpyAsync(points_host, x.qp_out, 7 * (size_t)x.n_qp_total * sizeof(double),
                                cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    return PG_OK;
}

int pg_write_vtk(pg_ctx* c, const char* path, double t) {
    PG_GUARD_CTX(c);
    if (!path) { set_error("pg_write_vtk: null path"); return PG_ERR_ARG; }
    try {
        return write_vtk(c->c, path, t);
    } catch (const std::exception& ex) {
        set_error(std::string("pg_write_vtk: host exception: ") + ex.what());
        return PG_ERR_ARG;
    }
}

int pg_write_cohesive_openings(pg_ctx* c, const char* path) {
    PG_GUARD_CTX(c);
    if (!path) { set_error("pg_write_cohesive_openings: null path"); return PG_ERR_ARG; }
    try {
        return write_cohesive_openings(c->c, path);
    } catch (const std::exception& ex) {
        set_error(std::string("pg_write_cohesive_openings: host exception: ") + ex.what());
        return PG_ERR_ARG;
    }
}

int pg_new_load_step(pg_ctx* c, double t_frac) {
    PG_GUARD_CTX(c);
    c->c.t_frac = t_frac;
    set_prescribed(c->c, t_frac, c->c.stream);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int pg_commit_isv(pg_ctx* c) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (x.n_coh_qp > 0)
        PG_CUDA(cudaMemcpyAsync(x.isv_c, x.isv_t, (size_t)x.n_coh_qp * sizeof(double), cudaMemcpyDeviceToDevice, x.stream));
    return PG_OK;
}

int pg_ctx_device_arrays(pg_ctx* c, double** K, double** U, double** F_int, double** isv_committed, double** isv_trial) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (K) *K = x.K;
    if (U) *U = x.U;
    if (F_int) *F_int = x.F;
    if (isv_committed) *isv_committed = x.isv_c;
    if (isv_trial) *isv_trial = x.isv_t;
    return PG_OK;
}

void pg_solver_cfg_default(pg_solver_cfg* cfg) {
    if (!cfg) return;
    cfg->krylov = PG_KRYLOV_CG;
    cfg->precond = PG_PREC_BLOCK_JACOBI;
    cfg->precision = PG_PRECISION_FP64;
    cfg->rtol = 1e-8;
    cfg->max_iter = 200000;
    cfg->inner_rtol = 1e-4;
    cfg->max_refine = 50;
    cfg->gmres_restart = 60;
    cfg->check_every = 64;
    cfg->inclusion_modes = 0;
    cfg->deterministic = 1;
}

int pg_solve_linear(pg_ctx* c, const pg_solver_cfg* cfg_in, pg_solve_stats* stats) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    pg_solver_cfg cfg;
    if (cfg_in) cfg = *cfg_in;
    else pg_solver_cfg_default(&cfg);
    pg_solve_stats st{};
    cudaStream_t s = x.stream;
    set_prescribed(x, 1.0, s);
    if (!x.assembled) {
        const int rc = launch_assemble(x, x.U, 0.0, false, true, s);
        if (rc != PG_OK) return rc;
        x.assembled = true;
    }
    const int rc = solve_linear_system(x, cfg, st, s);
    if (stats) *stats = st;
    if (rc != PG_OK) return rc;
    if (st.status != PG_OK) {
        set_error(st.status == PG_ERR_BREAKDOWN ? "pg_solve_linear: Krylov breakdown"
                                                : "pg_solve_linear: iteration budget exhausted before the tolerance");
        return st.status;
    }
    return PG_OK;
}

int pg_get_matrix(pg_ctx* c, double* vals_host) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!vals_host) { set_error("pg_get_matrix: null output"); return PG_ERR_ARG; }
    PG_CUDA(cudaStreamSynchronize(x.stream));
    PG_CUDA(cudaMemcpy(vals_host, x.K, 4 * (size_t)x.n_blocks * sizeof(double), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_get_vector(pg_ctx* c, int32_t which, double* out) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!out) { set_error("pg_get_vector: null output"); return PG_ERR_ARG; }
    const double* src = which == 0 ? x.U : which == 1 ? x.F : which == 2 ? x.r : nullptr;
    if (!src) { set_error("pg_get_vector: unknown vector"); return PG_ERR_ARG; }
    PG_CUDA(cudaStreamSynchronize(x.stream));
    PG_CUDA(cudaMemcpy(out, src, (size_t)x.n_dof * sizeof(double), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_set_vector(pg_ctx* c, int32_t which, const double* in) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!in) { set_error("pg_set_vector: null input"); return PG_ERR_ARG; }
    double* dst = which == 0 ? x.U : which == 1 ? x.F : nullptr;
    if (!dst) { set_error("pg_set_vector: unknown vector"); return PG_ERR_ARG; }
    PG_CUDA(cudaStreamSynchronize(x.stream));
    PG_CUDA(h2d_sync(dst, in, (size_t)x.n_dof * sizeof(double)));
    return PG_OK;
}

int pg_get_isv(pg_ctx* c, int32_t committed, double* out) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!out) { set_error("pg_get_isv: null output"); return PG_ERR_ARG; }
    if (x.n_coh_qp == 0) return PG_OK;
    PG_CUDA(cudaStreamSynchronize(x.stream));
    PG_CUDA(cudaMemcpy(out, committed ? x.isv_c : x.isv_t, (size_t)x.n_coh_qp * sizeof(double), cudaMemcpyDeviceToHost));
    return PG_OK;
}

int pg_assembly_timing(pg_ctx* c, int32_t enable, float* ms_rows, float* ms_cut) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (ms_rows || ms_cut) {
        if (!x.timing) { set_error("pg_assembly_timing: timing was not enabled"); return PG_ERR_STATE; }
        PG_CUDA(cudaEventSynchronize(x.ea2));
        float a = 0.f, b = 0.f;
        if (x.timing_split) {
            PG_CUDA(cudaEventElapsedTime(&a, x.ea0, x.ea1));
            PG_CUDA(cudaEventElapsedTime(&b, x.ea1, x.ea2));
        } else {
            PG_CUDA(cudaEventElapsedTime(&a, x.ea0, x.ea2));
        }
        if (ms_rows) *ms_rows = a;
        if (ms_cut) *ms_cut = b;
    }
    if (enable < 0 || enable > 2) { set_error("pg_assembly_timing: enable is 0, 1 or 2"); return PG_ERR_ARG; }
    x.timing = enable != 0;
    x.timing_split = enable == 1;
    return PG_OK;
}

int pg_set_isv(pg_ctx* c, int32_t committed, const double* in) {
    PG_GUARD_CTX(c);
    Ctx& x = c->c;
    if (!in) { set_error("pg_set_isv: null input"); return PG_ERR_ARG; }
    if (x.n_coh_qp == 0) return PG_OK;
    PG_CUDA(cudaStreamSynchronize(x.stream));
    PG_CUDA(h2d_sync(committed ? x.isv_c : x.isv_t, in, (size_t)x.n_coh_qp * sizeof(double)));
    return PG_OK;
}

}  // extern "C"
