// IGFEM preprocessing and sparsity on the GPU: the device counterpart of
// build_mesh (igfem_host.cpp), producing the same enriched mesh, DOF maps and
// block-CSR pattern bit for bit.
//
// Reference steps (PIGFEM 4.6.1, paths relative to PIGFEM4.6.1/):
//   Mesh::generate_mesh (TRI3)          src/Mesh.cpp:191-405
//   Mesh::analyze_nodes / detect_node   src/Mesh.cpp:2676-2714, 2838-2918
//   Tri3::detection (cut templates)     src/tri3.cpp:287-541
//   Mesh::analyze_elements              src/Mesh.cpp:2922-3027
//   Mesh::add_enrichments (serial)      src/Mesh.cpp:3038-3202, 3600-3660
//   Inclusion::find_intersection        src/Inclusion.cpp:32-128
//   DofObject::distribute_dofs          src/DofObject.cpp:241-386
//   Solver::preallocate_matrix          src/Solver.cpp:365-441, 723-829
//
// This file is compiled without FMA contraction (-fmad=false): every FP64
// operation rounds on its own, as the host builder's do, so coordinates,
// level sets and intersection points come out identical.  Division and
// square root are IEEE-rounded on both sides.
//
// Work per step: one thread per regular node (coordinates, detection), per
// element (template), per grid edge slot (enrichment numbering: the
// reference's std::set<((n0, n1), inclusion)> order is the order of the
// edge slots, four per node, so a scan over them numbers the enrichment
// nodes), per enrichment node (edge-circle root), per node row (pattern
// counts, then columns) and per cut element (slot tables).  Nodes that sit
// on an interface are moved by the node-moving rule on the host, in node
// order, as the reference does it: the rule reads the already-moved
// coordinates of lower-numbered nodes, and such nodes are few.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "pg_internal.cuh"

namespace pgb {
namespace {

constexpr int kThreadsMesh = 256;
inline int nb_mesh(long long n) { return (int)((n + kThreadsMesh - 1) / kThreadsMesh); }

// ---------------------------------------------------------------------------
// Exclusive scan of n ints in place (three launches: block scans, a scan of
// the block totals in one CTA, the block offsets added); returns the total.
// ---------------------------------------------------------------------------
constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(int* v, long long n, int* block_sum) {
    __shared__ int s[kScanBlock];
    const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
    const int x = i < n ? v[i] : 0;
    s[threadIdx.x] = x;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    if (i < n) v[i] = s[threadIdx.x] - x;
    if (threadIdx.x == kScanBlock - 1) block_sum[blockIdx.x] = s[threadIdx.x];
}

// one CTA: exclusive scan of the block totals (sequential chunks per thread)
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int* bs, int nblocks, int* total) {
    __shared__ int s[kScanBlock];
    const int per = (nblocks + kScanBlock - 1) / kScanBlock;
    const int b0 = threadIdx.x * per, b1 = min(nblocks, b0 + per);
    int local = 0;
    for (int b = b0; b < b1; ++b) local += bs[b];
    s[threadIdx.x] = local;
    __syncthreads();
    for (int off = 1; off < kScanBlock; off <<= 1) {
        const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    int run = s[threadIdx.x] - local;
    for (int b = b0; b < b1; ++b) {
        const int x = bs[b];
        bs[b] = run;
        run += x;
    }
    if (threadIdx.x == kScanBlock - 1) *total = s[threadIdx.x];
}

__global__ void k_scan_add(int* v, long long n, const int* bs) {
    const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n) v[i] += bs[blockIdx.x];
}

// Scratch owned by one device build: freed on every exit path.
// Scratch of one build, stream-ordered on the build's stream: many builds
// on host threads then run side by side (a plain cudaFree would synchronise
// the whole device at the end of each).
struct DevScratch {
    cudaStream_t s;
    std::vector<void*> owned;
    explicit DevScratch(cudaStream_t st) : s(st) {}
    ~DevScratch() {
        for (void* p : owned) cudaFreeAsync(p, s);
    }
    template <typename T>
    cudaError_t alloc(T** p, size_t n) {
        *p = nullptr;
        const cudaError_t e = cudaMallocAsync((void**)p, std::max<size_t>(1, n) * sizeof(T), s);
        if (e == cudaSuccess) owned.push_back(*p);
        return e;
    }
};

cudaError_t exclusive_scan(DevScratch& S, int* v, long long n, int& total, cudaStream_t s) {
    const int nblocks = (int)((n + kScanBlock - 1) / kScanBlock);
    int* bs = nullptr;
    int* tot = nullptr;
    cudaError_t e = S.alloc(&bs, nblocks);
    if (e == cudaSuccess) e = S.alloc(&tot, 1);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        k_scan_blocks<<<nblocks, kScanBlock, 0, s>>>(v, n, bs);
        k_scan_sums<<<1, kScanBlock, 0, s>>>(bs, nblocks, tot);
        k_scan_add<<<nblocks, kScanBlock, 0, s>>>(v, n, bs);
    } else {
        cudaMemsetAsync(tot, 0, sizeof(int), s);
    }
    e = cudaMemcpyAsync(&total, tot, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

// ---------------------------------------------------------------------------
// Geometry of the structured grid
// ---------------------------------------------------------------------------
struct GridDesc {
    int nx, ny, NX1;
    double x0, y0, hx, hy;
};

// vertices of element e (2 per cell, diagonal alternating with (i + j) % 2;
// Mesh.cpp:368-405, as the host builder lays them out)
__device__ __forceinline__ void elem_nodes(const GridDesc& g, int e, int n[3]) {
    const int cell = e >> 1, t = e & 1;
    const int i = cell % g.nx, j = cell / g.nx;
    const int n00 = i + j * g.NX1, n10 = n00 + 1, n01 = n00 + g.NX1, n11 = n01 + 1;
    if (((i + j) & 1) == 0) {
        if (t == 0) { n[0] = n00; n[1] = n10; n[2] = n11; }
        else { n[0] = n00; n[1] = n11; n[2] = n01; }
    } else {
        if (t == 0) { n[0] = n00; n[1] = n10; n[2] = n01; }
        else { n[0] = n10; n[1] = n11; n[2] = n01; }
    }
}

struct DevInclusion {
    double cx, cy, r;
    int mat;
};

// Regular nodes: coordinates and detection (Mesh.cpp:2838-2918) without the
// node-moving rule: a node on an interface (|level set| <= 1e-12) is
// flagged (detect = -2) for the host to move in node order.
__global__ void k_mesh_nodes(GridDesc g, const DevInclusion* __restrict__ inc, int ninc, double* x, double* y,
                             int* detect, int* n_flagged) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.NX1 * (g.ny + 1)) return;
    const int i = n % g.NX1, j = n / g.NX1;
    const double px = g.x0 + i * g.hx, py = g.y0 + j * g.hy;
    x[n] = px;
    y[n] = py;
    int result = -1;
    for (int k = ninc - 1; k >= 0; --k) {
        const DevInclusion c = inc[k];
        if (!(c.cx - c.r <= px && c.cy - c.r <= py && px <= c.cx + c.r && py <= c.cy + c.r)) continue;
        const double dx = px - c.cx, dy = py - c.cy;
        const double val = (sqrt(dx * dx + dy * dy) - c.r) / c.r;
        const double eps = 1e-12;
        if (val > eps) continue;
        if (val < -eps) { result = k; break; }
        result = -2;  // on the interface: the host applies the moving rule
        atomicAdd(n_flagged, 1);
        break;
    }
    detect[n] = result;
}

// Template choice from the three nodal detection values (-1 = matrix),
// the case analysis of Tri3::detection (tri3.cpp:287-541) as choose_template
// states it on the host.  -1: uncut; -2: not a case the templates cover.
__device__ int choose_template_dev(const int d[3], bool cohesive) {
    int v0 = d[0], v1 = d[1], v2 = d[2];
    // sort three values
    if (v0 > v1) { const int t = v0; v0 = v1; v1 = t; }
    if (v1 > v2) { const int t = v1; v1 = v2; v2 = t; }
    if (v0 > v1) { const int t = v0; v0 = v1; v1 = t; }
    const int n_unique = 1 + (v1 != v0) + (v2 != v1);
    if (n_unique == 1) return -1;
    const bool e01 = d[0] == d[1], e02 = d[0] == d[2], e12 = d[1] == d[2];
    const int base = cohesive ? 10 : 0;
    if (n_unique == 2) {
        int k;
        if (e12) k = 0;
        else if (e02) k = 1;
        else if (e01) k = 2;
        else return -2;
        if (v0 < 0) {
            if (!cohesive) return k;
            const int other = (k + 1) % 3;
            return d[k] < d[other] ? 10 + k : 13 + k;
        }
        return base + (cohesive ? 6 : 3) + k;
    }
    if (v0 < 0) {
        const int k = d[0] < 0 ? 0 : (d[1] < 0 ? 1 : 2);
        return base + (cohesive ? 9 : 6) + k;
    }
    return cohesive ? 22 : 9;
}

// Elements: connectivity, template, material of an uncut element, cut flag
// (elem_cut holds 1 / 0 here; the scan turns it into the cut index).
__global__ void k_mesh_elems(GridDesc g, const int* __restrict__ detect, const DevInclusion* __restrict__ inc,
                             int matrix_mat, bool cohesive, int* conn, int* elem_mat, int* elem_tmpl, int* cut_flag,
                             int* err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 2 * g.nx * g.ny) return;
    int n[3];
    elem_nodes(g, e, n);
    int d[3];
    for (int v = 0; v < 3; ++v) {
        conn[3 * (size_t)e + v] = n[v];
        d[v] = detect[n[v]];
    }
    const int t = choose_template_dev(d, cohesive);
    if (t == -2) atomicExch(err, 1);
    elem_tmpl[e] = t;
    cut_flag[e] = t >= 0 ? 1 : 0;
    elem_mat[e] = (t < 0 && d[0] != -1) ? inc[d[0]].mat : matrix_mat;
}


// Template data the device steps read (restated from cut_template()).
struct MeshTemplate {
    int n_cut_edges, n_enr, n_child, n_coh;
    int cut_edge[6];
    int enr_inc_node[6];
    int child_mat_node[kMaxChildren];
};
__constant__ MeshTemplate c_mtmpl[32];
__constant__ int c_edge_nodes[3][2] = {{0, 1}, {1, 2}, {2, 0}};  // Tri3::e_n_map (tri3.cpp:21-26)

// Edge slot of the grid edge (a, b), a < b: four per node a, in the order of
// b (right, upper-left diagonal, up, upper-right diagonal), so that slot
// order is the reference's (n0, n1) set order.
__device__ __forceinline__ long long edge_slot(const GridDesc& g, int a, int b) {
    const int d = b - a;
    const int dir = d == 1 ? 0 : (d == g.NX1 - 1 ? 1 : (d == g.NX1 ? 2 : 3));
    return 4LL * a + dir;
}

// Cut elements (cut order = element order): their arrays, and each cut-edge
// slot's inclusion marked on its grid edge slot.  An edge marked with two
// different inclusions is a case this builder does not number (err bit 2).
__global__ void k_mesh_cut(GridDesc g, int n_elem, const int* __restrict__ cut_idx, const int* __restrict__ cut_flag,
                           const int* __restrict__ elem_tmpl, const int* __restrict__ conn,
                           const int* __restrict__ detect, const DevInclusion* __restrict__ inc,
                           const int* __restrict__ elem_mat, int* cut_elem, int* cut_tmpl, int* cut_child_mat,
                           int* cut_coh_mat, int* slot_inc, int* coh_count, int* edge_inc, int* err) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elem || !cut_flag[e]) return;
    const int c = cut_idx[e];
    const int t = elem_tmpl[e];
    const MeshTemplate& T = c_mtmpl[t];
    cut_elem[c] = e;
    cut_tmpl[c] = t;
    int n[3], d[3], dmax = -1;
    for (int v = 0; v < 3; ++v) {
        n[v] = conn[3 * (size_t)e + v];
        d[v] = detect[n[v]];
        dmax = max(dmax, d[v]);
    }
    for (int k = 0; k < kMaxChildren; ++k) {
        int mat = -1;
        if (k < T.n_child) {
            const int nd = T.child_mat_node[k];
            mat = (nd < 0 || d[nd] < 0) ? elem_mat[e] : inc[d[nd]].mat;
        }
        cut_child_mat[(size_t)kMaxChildren * c + k] = mat;
    }
    for (int k = 0; k < kMaxCoh; ++k) cut_coh_mat[(size_t)kMaxCoh * c + k] = k < T.n_coh ? 0 : -1;
    coh_count[c] = 2 * T.n_coh;
    for (int s = 0; s < 6; ++s) slot_inc[6 * (size_t)c + s] = -1;
    for (int s = 0; s < T.n_cut_edges; ++s) {
        const int ic = T.enr_inc_node[s] < 0 ? dmax : d[T.enr_inc_node[s]];
        slot_inc[6 * (size_t)c + s] = ic;
        int a = n[c_edge_nodes[T.cut_edge[s]][0]], b = n[c_edge_nodes[T.cut_edge[s]][1]];
        if (a > b) { const int tt = a; a = b; b = tt; }
        const int old = atomicCAS(&edge_inc[edge_slot(g, a, b)], -1, ic);
        if (old != -1 && old != ic) atomicOr(err, 2);
    }
}

// edge slots carrying an inclusion: 1, others 0 (scanned into the numbering)
__global__ void k_edge_flags(long long n_slots, const int* __restrict__ edge_inc, int* flag) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_slots) flag[i] = edge_inc[i] >= 0 ? 1 : 0;
}

// Point on the edge p0 -> p1 where the circle is crossed: the root in [0, 1]
// of f(a) = |p0 + a (p1 - p0) - c|^2 / r^2 - 1, the level set the reference
// brackets and solves iteratively (Inclusion.cpp:32-128); the same closed
// form with two Newton steps as the host builder's circle_edge_root, op for
// op.
__device__ bool circle_edge_root_dev(double x0, double y0, double x1, double y1, const DevInclusion& inc,
                                     double& alpha) {
    const double g0x = (x0 + 0.0 * (x1 - x0) - inc.cx) / inc.r, g0y = (y0 + 0.0 * (y1 - y0) - inc.cy) / inc.r;
    const double g1x = (x0 + 1.0 * (x1 - x0) - inc.cx) / inc.r, g1y = (y0 + 1.0 * (y1 - y0) - inc.cy) / inc.r;
    const double f0 = g0x * g0x + g0y * g0y - 1.0, f1 = g1x * g1x + g1y * g1y - 1.0;
    if (f0 * f1 >= 0.0) return false;
    const double dx = (x1 - x0) / inc.r, dy = (y1 - y0) / inc.r;
    const double ex = (x0 - inc.cx) / inc.r, ey = (y0 - inc.cy) / inc.r;
    const double qa = dx * dx + dy * dy;
    const double qb = 2.0 * (ex * dx + ey * dy);
    const double qc = ex * ex + ey * ey - 1.0;
    const double dr = qb * qb - 4.0 * qa * qc;
    const double disc = dr < 0.0 ? 0.0 : dr;
    const double q = -0.5 * (qb + copysign(sqrt(disc), qb));
    const double r1 = q / qa, r2 = (q != 0.0) ? qc / q : r1;
    double a = (r1 >= 0.0 && r1 <= 1.0) ? r1 : r2;
    if (!(a >= 0.0 && a <= 1.0)) {
        const double lo = a < 0.0 ? 0.0 : a;
        a = 1.0 < lo ? 1.0 : lo;
    }
    for (int it = 0; it < 2; ++it) {
        const double gx = ex + a * dx, gy = ey + a * dy;
        const double fa = gx * gx + gy * gy - 1.0;
        const double dfa = 2.0 * (gx * dx + gy * dy);
        if (dfa == 0.0) break;
        const double an = a - fa / dfa;
        if (!(an >= 0.0 && an <= 1.0)) break;
        a = an;
    }
    alpha = a;
    return true;
}

// Enrichment nodes, one thread per numbered edge slot: edge, inclusion, and
// the intersection point (snapped onto an end node within rounding, as the
// host builder does), with the cohesive mirror copy at + n_initial.
__global__ void k_mesh_enr(GridDesc g, long long n_slots, const int* __restrict__ edge_inc,
                           const int* __restrict__ enr_idx, const DevInclusion* __restrict__ inc, int n_reg,
                           int n_init, bool cohesive, double* x, double* y, int* enr_edge, int* enr_inc, int* err) {
    const long long sl = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= n_slots) return;
    const int ic = edge_inc[sl];
    if (ic < 0) return;
    const int k = enr_idx[sl];
    const int a = (int)(sl >> 2), dir = (int)(sl & 3);
    const int b = a + (dir == 0 ? 1 : dir == 1 ? g.NX1 - 1 : dir == 2 ? g.NX1 : g.NX1 + 1);
    const double xa = x[a], ya = y[a], xb = x[b], yb = y[b];
    double alpha;
    if (!circle_edge_root_dev(xa, ya, xb, yb, inc[ic], alpha)) {
        atomicOr(err, 4);
        return;
    }
    double ex = xa + alpha * (xb - xa);
    double ey = ya + alpha * (yb - ya);
    const double tol = 8.0 * 2.220446049250313080847263336181640625e-16 *
                       (fabs(xb - xa) + fabs(yb - ya) + fabs(xb) + fabs(yb));
    if (fabs(ex - xa) + fabs(ey - ya) <= tol) { ex = xa; ey = ya; }
    if (fabs(ex - xb) + fabs(ey - yb) <= tol) { ex = xb; ey = yb; }
    for (int copy = 0; copy < (cohesive ? 2 : 1); ++copy) {
        const int idx = k + copy * n_init;
        x[n_reg + idx] = ex;
        y[n_reg + idx] = ey;
        enr_edge[2 * idx] = a;
        enr_edge[2 * idx + 1] = b;
        enr_inc[idx] = ic;
    }
}

// Each cut element's enrichment slots: the global node of every slot (the
// mirror slots of cohesive meshes follow the lower-surface ones).
__global__ void k_mesh_cut_enr(GridDesc g, int n_cut, const int* __restrict__ cut_elem, const int* __restrict__ cut_tmpl,
                               const int* __restrict__ conn, const int* __restrict__ slot_inc,
                               const int* __restrict__ edge_inc, const int* __restrict__ enr_idx, int n_reg,
                               int n_init, bool cohesive, int* cut_enr, int* err) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cut) return;
    const int e = cut_elem[c];
    const MeshTemplate& T = c_mtmpl[cut_tmpl[c]];
    int* out = cut_enr + (size_t)kMaxEnr * c;
    for (int s = 0; s < kMaxEnr; ++s) out[s] = -1;
    for (int s = 0; s < T.n_cut_edges; ++s) {
        int a = conn[3 * (size_t)e + c_edge_nodes[T.cut_edge[s]][0]], b = conn[3 * (size_t)e + c_edge_nodes[T.cut_edge[s]][1]];
        if (a > b) { const int tt = a; a = b; b = tt; }
        const long long sl = edge_slot(g, a, b);
        if (edge_inc[sl] != slot_inc[6 * (size_t)c + s]) { atomicOr(err, 2); continue; }
        const int k = enr_idx[sl];
        out[s] = n_reg + k;
        if (cohesive) out[s + T.n_cut_edges] = n_reg + k + n_init;
    }
}


// Grid neighbours of node (gi, gj) in its row, bits d = 3 (dy + 1) + (dx + 1)
// (the node itself at bit 4): axis neighbours inside the grid, diagonal
// ones too for even nodes (the only ones a cell diagonal passes through).
__device__ __forceinline__ unsigned nbr_mask(int gi, int gj, int nx, int ny) {
    const bool even = ((gi + gj) & 1) == 0;
    const bool w = gi > 0, e = gi < nx, s = gj > 0, n = gj < ny;
    return (s && even && w ? 1u : 0u) | (s ? 2u : 0u) | (s && even && e ? 4u : 0u) | (w ? 8u : 0u) | 16u |
           (e ? 32u : 0u) | (n && even && w ? 64u : 0u) | (n ? 128u : 0u) | (n && even && e ? 256u : 0u);
}

constexpr int kRowCap = 112;  // columns of one pattern row gathered before sorting

struct RowArgs {
    GridDesc g;
    int n_reg, n_nodes, n_init;
    const int* __restrict__ elem_cut;
    const int* __restrict__ cut_tmpl;
    const int* __restrict__ cut_enr;
    const int* __restrict__ conn;
    const int* __restrict__ enr_edge;
    const int* __restrict__ cut_elem;
};

__device__ __forceinline__ void push_unique(int* v, int& n, int x) {
    for (int i = 0; i < n; ++i)
        if (v[i] == x) return;
    if (n < kRowCap) v[n++] = x;
}

// the local node list of cut element c: 3 parents, then its enrichment slots
__device__ __forceinline__ int cut_local_nodes(const RowArgs& a, int c, int* L) {
    const int e = a.cut_elem[c];
    const int nl = 3 + c_mtmpl[a.cut_tmpl[c]].n_enr;
    for (int v = 0; v < 3; ++v) L[v] = a.conn[3 * (size_t)e + v];
    for (int s = 0; s < nl - 3; ++s) L[3 + s] = a.cut_enr[(size_t)kMaxEnr * c + s];
    return nl;
}

// Columns of row n, ascending, the way the host builder's adjacency sets
// collect them: a regular node's grid neighbours and itself (every element
// around it, cut or not, contributes its vertices) then the enrichment nodes
// of the cut elements around it; an enrichment node's union of the local
// node lists of the cut elements holding it.  Returns the count; v is
// sorted.  *overflow is set past kRowCap columns.
__device__ int row_columns(const RowArgs& a, int n, int* v, int* overflow) {
    const GridDesc& g = a.g;
    int cnt = 0;
    if (n < a.n_reg) {
        const int gi = n % g.NX1, gj = n / g.NX1;
        const unsigned mask = nbr_mask(gi, gj, g.nx, g.ny);
        int enr[kRowCap];
        int ne = 0;
        for (int oy = 0; oy < 2; ++oy)
            for (int ox = 0; ox < 2; ++ox) {
                const int ci = gi - 1 + ox, cj = gj - 1 + oy;
                if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny) continue;
                for (int t = 0; t < 2; ++t) {
                    const int e = 2 * (ci + cj * g.nx) + t;
                    const int c = a.elem_cut[e];
                    if (c < 0) continue;
                    int L[kMaxElemNodes];
                    const int nl = cut_local_nodes(a, c, L);
                    if (L[0] != n && L[1] != n && L[2] != n) continue;
                    for (int k = 3; k < nl; ++k) push_unique(enr, ne, L[k]);
                }
            }
        for (int d = 0; d < 9; ++d)
            if (mask & (1u << d)) v[cnt++] = n + (d % 3 - 1) + (d / 3 - 1) * g.NX1;
        // insertion sort of the enrichment columns (all beyond the regular ones)
        for (int i = 1; i < ne; ++i) {
            const int x = enr[i];
            int j = i - 1;
            while (j >= 0 && enr[j] > x) { enr[j + 1] = enr[j]; --j; }
            enr[j + 1] = x;
        }
        if (cnt + ne > kRowCap) { atomicOr(overflow, 1); ne = kRowCap - cnt; }
        for (int i = 0; i < ne; ++i) v[cnt++] = enr[i];
        return cnt;
    }
    // enrichment node: its edge's elements that hold it
    const int idx = n - a.n_reg;
    const int ea = a.enr_edge[2 * idx], eb = a.enr_edge[2 * idx + 1];
    const int gi = ea % g.NX1, gj = ea / g.NX1;
    push_unique(v, cnt, n);
    for (int oy = 0; oy < 2; ++oy)
        for (int ox = 0; ox < 2; ++ox) {
            const int ci = gi - 1 + ox, cj = gj - 1 + oy;
            if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny) continue;
            for (int t = 0; t < 2; ++t) {
                const int e = 2 * (ci + cj * g.nx) + t;
                const int c = a.elem_cut[e];
                if (c < 0) continue;
                int L[kMaxElemNodes];
                const int nl = cut_local_nodes(a, c, L);
                bool holds = false;
                for (int k = 3; k < nl; ++k) holds |= L[k] == n;
                if (!holds) continue;
                for (int k = 0; k < nl; ++k) push_unique(v, cnt, L[k]);
            }
        }
    (void)eb;
    for (int i = 1; i < cnt; ++i) {
        const int x = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > x) { v[j + 1] = v[j]; --j; }
        v[j + 1] = x;
    }
    if (cnt >= kRowCap) atomicOr(overflow, 1);
    return cnt;
}

__global__ void k_row_counts(RowArgs a, int* counts, int* overflow) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.n_nodes) return;
    int v[kRowCap];
    counts[n] = row_columns(a, n, v, overflow);
}

__global__ void k_row_fill(RowArgs a, const int* __restrict__ row_ptr, int* col, int* diag, int* overflow) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= a.n_nodes) return;
    int v[kRowCap];
    const int cnt = row_columns(a, n, v, overflow);
    const int q0 = row_ptr[n];
    for (int i = 0; i < cnt; ++i) {
        col[q0 + i] = v[i];
        if (v[i] == n) diag[n] = q0 + i;
    }
}

// Per node: the uncut elements around it in element order, packed
// (element << 2) | local vertex (none for enrichment nodes).  Pass 0 counts,
// pass 1 fills.
__global__ void k_node_elems(GridDesc g, int n_nodes, int n_reg, const int* __restrict__ elem_cut,
                             const int* __restrict__ conn, const int* __restrict__ ptr, int* out, int pass) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= n_nodes) return;
    int cnt = 0;
    if (n < n_reg) {
        const int gi = n % g.NX1, gj = n / g.NX1;
        int q = pass ? ptr[n] : 0;
        for (int oy = 0; oy < 2; ++oy)
            for (int ox = 0; ox < 2; ++ox) {
                const int ci = gi - 1 + ox, cj = gj - 1 + oy;
                if (ci < 0 || ci >= g.nx || cj < 0 || cj >= g.ny) continue;
                for (int t = 0; t < 2; ++t) {
                    const int e = 2 * (ci + cj * g.nx) + t;
                    if (elem_cut[e] >= 0) continue;
                    for (int v = 0; v < 3; ++v)
                        if (conn[3 * (size_t)e + v] == n) {
                            if (pass) out[q++] = (e << 2) | v;
                            ++cnt;
                        }
                }
            }
    }
    if (!pass) out[n] = cnt;
}

// Per cut element: the block slot of every local pair (a, b) (binary search
// in row L[a]); kMaxElemNodes^2 entries, -1 unused (cleared beforehand).
__global__ void k_cut_slots(RowArgs a, int n_cut, const int* __restrict__ row_ptr, const int* __restrict__ col,
                            int* cut_slot) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cut) return;
    int L[kMaxElemNodes];
    const int nl = cut_local_nodes(a, c, L);
    constexpr int S = kMaxElemNodes;
    for (int i = 0; i < nl; ++i) {
        const int q0 = row_ptr[L[i]], q1 = row_ptr[L[i] + 1];
        for (int j = 0; j < nl; ++j) {
            int lo = q0, hi = q1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (col[mid] < L[j]) lo = mid + 1;
                else hi = mid;
            }
            cut_slot[(size_t)c * S * S + i * S + j] = (lo < q1 && col[lo] == L[j]) ? lo : -1;
        }
    }
}

// Dirichlet data (Tests/Main.cpp:444-450): u_x = 0 on the left edge, u_x =
// app on the right edge, node 0 fixed in both directions; free_flag holds
// 1 for the free regular DOFs (scanned into the free-first numbering).
__global__ void k_dofs(GridDesc g, int n_dof, int n_reg, double app, uint8_t* fixed, double* ubar, int* free_flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_dof) return;
    const int n = i >> 1, d = i & 1;
    bool f = false;
    double u = 0.0;
    if (n < n_reg) {
        const int gi = n % g.NX1;
        if (d == 0 && gi == 0) f = true;
        if (d == 0 && gi == g.nx) { f = true; u = app; }
        if (n == 0) { f = true; u = 0.0; }
        free_flag[i] = f ? 0 : 1;
    }
    fixed[i] = f ? 1 : 0;
    ubar[i] = u;
}

// reference DOF numbers: free regular DOFs in order, enrichment DOFs after
// them, prescribed DOFs after all free ones (DofObject.cpp:241-386)
__global__ void k_ref_dof(int n_dof, int n_reg, int n_free, int n_reg_free, const uint8_t* __restrict__ fixed,
                          const int* __restrict__ free_idx, int* ref_dof) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_dof) return;
    if (i < 2 * n_reg) ref_dof[i] = fixed[i] ? n_free + (i - free_idx[i]) : free_idx[i];
    else ref_dof[i] = n_reg_free + (i - 2 * n_reg);
}


__global__ void k_elem_cut(int n_elem, const int* __restrict__ flag, const int* __restrict__ idx, int* elem_cut) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n_elem) elem_cut[e] = flag[e] ? idx[e] : -1;
}

void upload_mesh_templates() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);  // builds may run from several host threads
    if (dev >= 0 && dev < 64 && done[dev]) return;
    MeshTemplate t[32] = {};
    for (int i = 0; i < n_cut_templates() && i < 32; ++i) {
        const CutTemplate& T = cut_template(i);
        t[i].n_cut_edges = T.n_cut_edges;
        t[i].n_enr = T.n_enr;
        t[i].n_child = T.n_child;
        t[i].n_coh = T.n_coh;
        for (int k = 0; k < 6; ++k) {
            t[i].cut_edge[k] = T.cut_edge[k];
            t[i].enr_inc_node[k] = T.enr_inc_node[k];
        }
        for (int k = 0; k < kMaxChildren; ++k) t[i].child_mat_node[k] = T.child_mat_node[k];
    }
    cudaMemcpyToSymbol(c_mtmpl, t, sizeof(t));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

// The reference's node-moving rule (Mesh.cpp:2895-2918) for one node flagged
// on an interface, on the host, exactly as build_mesh applies it: the node
// moves by 5% of the edge to the first vertex of its first element along the
// outward normal, at most five times, rescanning the inclusions after every
// move.  Returns the detection value, or -2 when the node cannot be moved off.
int move_node_host(const RveSpec& spec, int nx, int n, std::vector<double>& x, std::vector<double>& y, int& n_moved) {
    const int NX1 = nx + 1, ninc = (int)spec.inclusions.size();
    // the lowest-numbered element holding n (the cells around it in index
    // order, t = 0 before t = 1) and its first vertex other than n
    const int gi = n % NX1, gj = n / NX1;
    int other = -1;
    for (int oy = 0; oy < 2 && other < 0; ++oy)
        for (int ox = 0; ox < 2 && other < 0; ++ox) {
            const int ci = gi - 1 + ox, cj = gj - 1 + oy;
            if (ci < 0 || ci >= nx || cj < 0 || cj >= spec.ny) continue;
            for (int t = 0; t < 2 && other < 0; ++t) {
                const int n00 = ci + cj * NX1, n10 = n00 + 1, n01 = n00 + NX1, n11 = n01 + 1;
                int v[3];
                if (((ci + cj) & 1) == 0) {
                    if (t == 0) { v[0] = n00; v[1] = n10; v[2] = n11; }
                    else { v[0] = n00; v[1] = n11; v[2] = n01; }
                } else {
                    if (t == 0) { v[0] = n00; v[1] = n10; v[2] = n01; }
                    else { v[0] = n10; v[1] = n11; v[2] = n01; }
                }
                if (v[0] == n || v[1] == n || v[2] == n) other = v[0] == n ? v[1] : v[0];
            }
        }
    int moved = 0, result = -1;
    for (int j = ninc - 1; j >= 0; --j) {
        const Inclusion& inc = spec.inclusions[j];
        const double px = x[n], py = y[n];
        if (!(inc.cx - inc.r <= px && inc.cy - inc.r <= py && px <= inc.cx + inc.r && py <= inc.cy + inc.r)) continue;
        const double dx = px - inc.cx, dy = py - inc.cy;
        const double val = (std::sqrt(dx * dx + dy * dy) - inc.r) / inc.r;
        const double eps = 1e-12;
        if (val > eps) continue;
        if (val < -eps) { result = j; break; }
        if (moved >= 5) return -3;
        const double nrm = std::sqrt(dx * dx + dy * dy);
        const double nxn = dx / nrm, nyn = dy / nrm;
        const double ox = x[other], oy = y[other];
        const double dist = 0.05 * std::sqrt((px - ox) * (px - ox) + (py - oy) * (py - oy) + 0.0);
        x[n] = px + dist * nxn;
        y[n] = py + dist * nyn;
        ++moved;
        ++n_moved;
        j = ninc;
    }
    return result;
}

template <typename T>
cudaError_t download(std::vector<T>& h, const T* d, size_t n, cudaStream_t s) {
    h.resize(n);
    if (n == 0) return cudaSuccess;
    return cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, s);
}


// ---------------------------------------------------------------------------
// Fold order of the cut elements' pair blocks (pg_assemble.cu), built on the
// GPU by a counting sort: every slot-table entry (class-ordered element oi,
// pair p = a nl + b) counts itself into its K slot and into its row node a;
// exclusive scans give every slot's and node's run; the entries scatter into
// their runs; each run is then put in entry order, so the result is the
// order (key, entry) a sort would give, the same on every run.
// ---------------------------------------------------------------------------
__global__ void k_fold_count(int nc, const int* __restrict__ sp, const int* __restrict__ sl,
                             const int* __restrict__ nodes, const uint8_t* __restrict__ node_enr, int* cntK,
                             uint8_t* cutK, int* cntF) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nc) return;
    const int s0 = sp[oi], np = sp[oi + 1] - s0;
    int nl = 0;
    while (nl * nl < np) ++nl;
    for (int p = 0; p < np; ++p) {
        const int a = p / nl, b = p - a * nl;
        const int na = nodes[(size_t)kCutNodeStride * oi + a], nb = nodes[(size_t)kCutNodeStride * oi + b];
        const int slot = sl[s0 + p];
        if (slot >= 0) {
            atomicAdd(&cntK[slot], 1);
            if (node_enr[na] || node_enr[nb]) cutK[slot] = 1;
        }
        atomicAdd(&cntF[na], 1);
    }
}

// runs: a key i is touched when start[i + 1] > start[i]; touched_idx holds
// the scan of those flags (its run number)
__global__ void k_fold_touched(long long n, const int* __restrict__ start, int* touched) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) touched[i] = start[i + 1] > start[i] ? 1 : 0;
}

template <typename KeyT>
__global__ void k_fold_runs(long long n, const int* __restrict__ start, const int* __restrict__ run_of,
                            const uint8_t* __restrict__ cut_only, KeyT* run_key, int* run_ptr) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || start[i + 1] == start[i]) return;
    const int r = run_of[i];
    run_key[r] = (KeyT)((KeyT)i << 1) | (KeyT)(cut_only[i] ? 1 : 0);
    run_ptr[r] = start[i];
}

__global__ void k_fold_scatter(int nc, const int* __restrict__ sp, const int* __restrict__ sl,
                               const int* __restrict__ nodes, const int* __restrict__ startK, int* fillK, int* tmpK,
                               const int* __restrict__ startF, int* fillF, int* tmpF) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= nc) return;
    const int s0 = sp[oi], np = sp[oi + 1] - s0;
    int nl = 0;
    while (nl * nl < np) ++nl;
    for (int p = 0; p < np; ++p) {
        const int a = p / nl;
        const int na = nodes[(size_t)kCutNodeStride * oi + a];
        const int slot = sl[s0 + p];
        if (slot >= 0) tmpK[startK[slot] + atomicAdd(&fillK[slot], 1)] = s0 + p;
        tmpF[startF[na] + atomicAdd(&fillF[na], 1)] = s0 + p;
    }
}

// one thread per K run: a run of one entry gives that entry its slot (the
// cut-element kernel adds it to K itself); the others are flagged for the fold
__global__ void k_fold_single(int nruns, const int* __restrict__ run_ptr, const int* __restrict__ tmp,
                              const long long* __restrict__ run_key, long long* kdir, int* multi) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const int i0 = run_ptr[r];
    const bool single = run_ptr[r + 1] - i0 == 1;
    if (single) kdir[tmp[i0]] = run_key[r];
    multi[r] = single ? 0 : 1;
}

// entries of the longer runs: kdir = -2 - (their fold position)
__global__ void k_fold_kdir_multi(int n, const int* __restrict__ kpos, long long* kdir) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n && kdir[e] == -1 && kpos[e] >= 0) kdir[e] = -2 - (long long)kpos[e];
}

__global__ void k_fold_multi(int nruns, const int* __restrict__ flag, const int* __restrict__ idx,
                             const long long* __restrict__ run_key, const int* __restrict__ run_ptr,
                             long long* m_key, int2* m_rng) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns || !flag[r]) return;
    m_key[idx[r]] = run_key[r];
    m_rng[idx[r]] = make_int2(run_ptr[r], run_ptr[r + 1]);
}

// one thread per run: its entries in entry order, and each entry's position
__global__ void k_fold_order(int nruns, const int* __restrict__ run_ptr, int* tmp, int* pos) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nruns) return;
    const int i0 = run_ptr[r], i1 = run_ptr[r + 1];
    for (int i = i0 + 1; i < i1; ++i) {
        const int x = tmp[i];
        int j = i - 1;
        while (j >= i0 && tmp[j] > x) { tmp[j + 1] = tmp[j]; --j; }
        tmp[j + 1] = x;
    }
    for (int i = i0; i < i1; ++i) pos[tmp[i]] = i;
}

}  // namespace

#define MESH_CUDA(call)                                                          \
    do {                                                                         \
        const cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) return cuda_fail(_e, "device mesh set-up: " #call); \
    } while (0)

int build_mesh_device(const RveSpec& spec, int device, HostMesh& m) {
    m = HostMesh();
    m.spec = spec;
    const int nx = spec.nx, ny = spec.ny;
    if (nx < 1 || ny < 1) { set_error("pg_mesh_build_device: mesh needs at least one element in each direction"); return PG_ERR_MESH; }
    if ((long long)(nx + 1) * (ny + 1) > (1ll << 28) || 2LL * nx * ny > (1ll << 29)) {
        set_error("pg_mesh_build_device: mesh too large");
        return PG_ERR_MESH;
    }
    if (spec.materials.empty() || spec.matrix_mat < 0 || spec.matrix_mat >= (int)spec.materials.size()) {
        set_error("pg_mesh_build_device: invalid matrix material");
        return PG_ERR_MESH;
    }
    for (const auto& inc : spec.inclusions)
        if (inc.r <= 0.0 || inc.mat < 0 || inc.mat >= (int)spec.materials.size()) {
            set_error("pg_mesh_build_device: invalid inclusion");
            return PG_ERR_MESH;
        }
    MESH_CUDA(cudaSetDevice(device));
    upload_mesh_templates();
    cudaStream_t s = nullptr;
    MESH_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    DevScratch S(s);

    GridDesc g;
    g.nx = nx;
    g.ny = ny;
    g.NX1 = nx + 1;
    g.x0 = spec.x0;
    g.y0 = spec.y0;
    g.hx = (spec.x1 - spec.x0) / nx;
    g.hy = (spec.y1 - spec.y0) / ny;
    const int n_reg = (nx + 1) * (ny + 1), n_elem = 2 * nx * ny;
    const int ninc = (int)spec.inclusions.size();
    m.n_reg = n_reg;
    m.n_elem = n_elem;
    m.grids.push_back({nx, ny, 0, 0, n_reg});

    // ---- nodes and their detection ----
    std::vector<DevInclusion> hinc(ninc);
    for (int k = 0; k < ninc; ++k)
        hinc[k] = {spec.inclusions[k].cx, spec.inclusions[k].cy, spec.inclusions[k].r, spec.inclusions[k].mat};
    DevInclusion* dinc;
    double *xr, *yr;
    int *detect, *counters;  // counters: [0] flagged nodes, [1] error bits
    MESH_CUDA(S.alloc(&dinc, ninc));
    MESH_CUDA(S.alloc(&xr, n_reg));
    MESH_CUDA(S.alloc(&yr, n_reg));
    MESH_CUDA(S.alloc(&detect, n_reg));
    MESH_CUDA(S.alloc(&counters, 2));
    if (ninc) MESH_CUDA(cudaMemcpyAsync(dinc, hinc.data(), ninc * sizeof(DevInclusion), cudaMemcpyHostToDevice, s));
    MESH_CUDA(cudaMemsetAsync(counters, 0, 2 * sizeof(int), s));
    k_mesh_nodes<<<nb_mesh(n_reg), kThreadsMesh, 0, s>>>(g, dinc, ninc, xr, yr, detect, counters);
    int hc[2] = {0, 0};
    MESH_CUDA(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, s));
    MESH_CUDA(cudaStreamSynchronize(s));
    if (hc[0] > 0) {
        // nodes on an interface: the moving rule, in node order, on the host
        MESH_CUDA(download(m.x, xr, n_reg, s));
        MESH_CUDA(download(m.y, yr, n_reg, s));
        MESH_CUDA(download(m.node_detect, detect, n_reg, s));
        MESH_CUDA(cudaStreamSynchronize(s));
        for (int n = 0; n < n_reg; ++n) {
            if (m.node_detect[n] != -2) continue;
            const int r = move_node_host(spec, nx, n, m.x, m.y, m.n_moved);
            if (r == -3) {
                set_error("pg_mesh_build_device: unable to move node " + std::to_string(n) + " off an inclusion surface");
                return PG_ERR_MESH;
            }
            m.node_detect[n] = r;
        }
        MESH_CUDA(cudaMemcpyAsync(xr, m.x.data(), n_reg * sizeof(double), cudaMemcpyHostToDevice, s));
        MESH_CUDA(cudaMemcpyAsync(yr, m.y.data(), n_reg * sizeof(double), cudaMemcpyHostToDevice, s));
        MESH_CUDA(cudaMemcpyAsync(detect, m.node_detect.data(), n_reg * sizeof(int), cudaMemcpyHostToDevice, s));
    }

    // ---- elements and templates ----
    int *conn, *elem_mat, *elem_tmpl, *cut_flag, *cut_idx, *elem_cut;
    MESH_CUDA(S.alloc(&conn, 3 * (size_t)n_elem));
    MESH_CUDA(S.alloc(&elem_mat, n_elem));
    MESH_CUDA(S.alloc(&elem_tmpl, n_elem));
    MESH_CUDA(S.alloc(&cut_flag, n_elem));
    MESH_CUDA(S.alloc(&cut_idx, n_elem));
    MESH_CUDA(S.alloc(&elem_cut, n_elem));
    k_mesh_elems<<<nb_mesh(n_elem), kThreadsMesh, 0, s>>>(g, detect, dinc, spec.matrix_mat, spec.cohesive, conn,
                                                          elem_mat, elem_tmpl, cut_flag, counters + 1);
    MESH_CUDA(cudaMemcpyAsync(cut_idx, cut_flag, n_elem * sizeof(int), cudaMemcpyDeviceToDevice, s));
    int n_cut = 0;
    MESH_CUDA(exclusive_scan(S, cut_idx, n_elem, n_cut, s));
    k_elem_cut<<<nb_mesh(n_elem), kThreadsMesh, 0, s>>>(n_elem, cut_flag, cut_idx, elem_cut);
    m.n_cut = n_cut;

    // ---- cut elements and their cut edges ----
    const long long n_slots = 4LL * n_reg;
    int *cut_elem, *cut_tmpl, *cut_child_mat, *cut_coh_mat, *slot_inc, *coh_count, *edge_inc, *enr_idx;
    MESH_CUDA(S.alloc(&cut_elem, n_cut));
    MESH_CUDA(S.alloc(&cut_tmpl, n_cut));
    MESH_CUDA(S.alloc(&cut_child_mat, (size_t)kMaxChildren * n_cut));
    MESH_CUDA(S.alloc(&cut_coh_mat, (size_t)kMaxCoh * n_cut));
    MESH_CUDA(S.alloc(&slot_inc, 6 * (size_t)n_cut));
    MESH_CUDA(S.alloc(&coh_count, n_cut + 1));
    MESH_CUDA(S.alloc(&edge_inc, n_slots));
    MESH_CUDA(S.alloc(&enr_idx, n_slots));
    MESH_CUDA(cudaMemsetAsync(edge_inc, 0xff, n_slots * sizeof(int), s));
    MESH_CUDA(cudaMemsetAsync(coh_count, 0, (n_cut + 1) * sizeof(int), s));
    k_mesh_cut<<<nb_mesh(n_elem), kThreadsMesh, 0, s>>>(g, n_elem, cut_idx, cut_flag, elem_tmpl, conn, detect, dinc,
                                                        elem_mat, cut_elem, cut_tmpl, cut_child_mat, cut_coh_mat,
                                                        slot_inc, coh_count, edge_inc, counters + 1);
    k_edge_flags<<<nb_mesh(n_slots), kThreadsMesh, 0, s>>>(n_slots, edge_inc, enr_idx);
    int n_init = 0;
    MESH_CUDA(exclusive_scan(S, enr_idx, n_slots, n_init, s));
    MESH_CUDA(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, s));
    MESH_CUDA(cudaStreamSynchronize(s));
    if (hc[1] & 1) { set_error("pg_mesh_build_device: triangle with one node separated in an unknown manner"); return PG_ERR_MESH; }
    if (hc[1] & 2) { set_error("pg_mesh_build_device: a grid edge cut by two inclusions (use pg_mesh_build)"); return PG_ERR_MESH; }
    m.n_enr_initial = n_init;
    m.n_enr = spec.cohesive ? 2 * n_init : n_init;
    const int nn = n_reg + m.n_enr;

    // ---- enrichment nodes ----
    double *x, *y;
    int *enr_edge, *enr_inc, *cut_enr;
    MESH_CUDA(S.alloc(&x, nn));
    MESH_CUDA(S.alloc(&y, nn));
    MESH_CUDA(S.alloc(&enr_edge, 2 * (size_t)m.n_enr));
    MESH_CUDA(S.alloc(&enr_inc, m.n_enr));
    MESH_CUDA(S.alloc(&cut_enr, (size_t)kMaxEnr * n_cut));
    MESH_CUDA(cudaMemcpyAsync(x, xr, n_reg * sizeof(double), cudaMemcpyDeviceToDevice, s));
    MESH_CUDA(cudaMemcpyAsync(y, yr, n_reg * sizeof(double), cudaMemcpyDeviceToDevice, s));
    k_mesh_enr<<<nb_mesh(n_slots), kThreadsMesh, 0, s>>>(g, n_slots, edge_inc, enr_idx, dinc, n_reg, n_init,
                                                         spec.cohesive, x, y, enr_edge, enr_inc, counters + 1);
    k_mesh_cut_enr<<<nb_mesh(n_cut), kThreadsMesh, 0, s>>>(g, n_cut, cut_elem, cut_tmpl, conn, slot_inc, edge_inc,
                                                           enr_idx, n_reg, n_init, spec.cohesive, cut_enr,
                                                           counters + 1);
    MESH_CUDA(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, s));
    MESH_CUDA(cudaStreamSynchronize(s));
    if (hc[1] & 4) { set_error("pg_mesh_build_device: no valid intersection on a cut edge"); return PG_ERR_MESH; }
    if (hc[1] & 2) { set_error("pg_mesh_build_device: cut edge without its enrichment node"); return PG_ERR_MESH; }

    // ---- Dirichlet data and the reference DOF numbering ----
    const int n_dof = 2 * nn;
    uint8_t* fixed;
    double* ubar;
    int *free_idx, *ref_dof;
    MESH_CUDA(S.alloc(&fixed, n_dof));
    MESH_CUDA(S.alloc(&ubar, n_dof));
    MESH_CUDA(S.alloc(&free_idx, 2 * (size_t)n_reg));
    MESH_CUDA(S.alloc(&ref_dof, n_dof));
    const double app = (spec.x1 - spec.x0) * spec.strain;
    k_dofs<<<nb_mesh(n_dof), kThreadsMesh, 0, s>>>(g, n_dof, n_reg, app, fixed, ubar, free_idx);
    int n_reg_free = 0;
    MESH_CUDA(exclusive_scan(S, free_idx, 2LL * n_reg, n_reg_free, s));
    m.n_free = n_reg_free + 2 * m.n_enr;
    k_ref_dof<<<nb_mesh(n_dof), kThreadsMesh, 0, s>>>(n_dof, n_reg, m.n_free, n_reg_free, fixed, free_idx, ref_dof);

    // ---- 2x2-block pattern, element lists, slot tables ----
    RowArgs ra;
    ra.g = g;
    ra.n_reg = n_reg;
    ra.n_nodes = nn;
    ra.n_init = n_init;
    ra.elem_cut = elem_cut;
    ra.cut_tmpl = cut_tmpl;
    ra.cut_enr = cut_enr;
    ra.conn = conn;
    ra.enr_edge = enr_edge;
    ra.cut_elem = cut_elem;
    int *row_ptr, *col, *diag, *ne_ptr, *ne_list, *cut_slot;
    MESH_CUDA(S.alloc(&row_ptr, nn + 1));
    MESH_CUDA(S.alloc(&diag, nn));
    MESH_CUDA(cudaMemsetAsync(row_ptr, 0, (nn + 1) * sizeof(int), s));
    k_row_counts<<<nb_mesh(nn), kThreadsMesh, 0, s>>>(ra, row_ptr, counters + 1);
    int nnzb = 0;
    MESH_CUDA(exclusive_scan(S, row_ptr, nn + 1LL, nnzb, s));
    MESH_CUDA(S.alloc(&col, nnzb));
    k_row_fill<<<nb_mesh(nn), kThreadsMesh, 0, s>>>(ra, row_ptr, col, diag, counters + 1);
    MESH_CUDA(S.alloc(&ne_ptr, nn + 1));
    MESH_CUDA(cudaMemsetAsync(ne_ptr, 0, (nn + 1) * sizeof(int), s));
    k_node_elems<<<nb_mesh(nn), kThreadsMesh, 0, s>>>(g, nn, n_reg, elem_cut, conn, nullptr, ne_ptr, 0);
    int n_ne = 0;
    MESH_CUDA(exclusive_scan(S, ne_ptr, nn + 1LL, n_ne, s));
    MESH_CUDA(S.alloc(&ne_list, n_ne));
    k_node_elems<<<nb_mesh(nn), kThreadsMesh, 0, s>>>(g, nn, n_reg, elem_cut, conn, ne_ptr, ne_list, 1);
    constexpr int SS = kMaxElemNodes * kMaxElemNodes;
    MESH_CUDA(S.alloc(&cut_slot, (size_t)SS * n_cut));
    MESH_CUDA(cudaMemsetAsync(cut_slot, 0xff, (size_t)SS * n_cut * sizeof(int), s));
    k_cut_slots<<<nb_mesh(n_cut), kThreadsMesh, 0, s>>>(ra, n_cut, row_ptr, col, cut_slot);
    int n_coh_qp = 0;
    MESH_CUDA(exclusive_scan(S, coh_count, n_cut + 1LL, n_coh_qp, s));
    m.n_coh_qp = n_coh_qp;
    MESH_CUDA(cudaMemcpyAsync(hc, counters, sizeof hc, cudaMemcpyDeviceToHost, s));
    MESH_CUDA(cudaStreamSynchronize(s));
    MESH_CUDA(cudaGetLastError());
    if (hc[1] & 1) { set_error("pg_mesh_build_device: a pattern row exceeds the builder's column capacity"); return PG_ERR_MESH; }

    // ---- the host copy every other part of the library reads ----
    MESH_CUDA(download(m.x, x, nn, s));
    MESH_CUDA(download(m.y, y, nn, s));
    MESH_CUDA(download(m.node_detect, detect, n_reg, s));
    MESH_CUDA(download(m.conn, conn, 3 * (size_t)n_elem, s));
    MESH_CUDA(download(m.elem_mat, elem_mat, n_elem, s));
    MESH_CUDA(download(m.elem_cut, elem_cut, n_elem, s));
    MESH_CUDA(download(m.cut_elem, cut_elem, n_cut, s));
    MESH_CUDA(download(m.cut_tmpl, cut_tmpl, n_cut, s));
    MESH_CUDA(download(m.cut_enr, cut_enr, (size_t)kMaxEnr * n_cut, s));
    MESH_CUDA(download(m.cut_child_mat, cut_child_mat, (size_t)kMaxChildren * n_cut, s));
    MESH_CUDA(download(m.cut_coh_mat, cut_coh_mat, (size_t)kMaxCoh * n_cut, s));
    MESH_CUDA(download(m.enr_edge, enr_edge, 2 * (size_t)m.n_enr, s));
    MESH_CUDA(download(m.enr_inc, enr_inc, m.n_enr, s));
    MESH_CUDA(download(m.fixed, fixed, n_dof, s));
    MESH_CUDA(download(m.ubar, ubar, n_dof, s));
    MESH_CUDA(download(m.ref_dof, ref_dof, n_dof, s));
    MESH_CUDA(download(m.row_ptr, row_ptr, nn + 1, s));
    MESH_CUDA(download(m.col, col, nnzb, s));
    MESH_CUDA(download(m.diag_slot, diag, nn, s));
    MESH_CUDA(download(m.ne_ptr, ne_ptr, nn + 1, s));
    MESH_CUDA(download(m.ne_list, ne_list, n_ne, s));
    MESH_CUDA(download(m.cut_slot, cut_slot, (size_t)SS * n_cut, s));
    MESH_CUDA(download(m.cut_coh_qp0, coh_count, n_cut, s));
    MESH_CUDA(cudaStreamSynchronize(s));
    return PG_OK;
}

}  // namespace pgb

namespace pgb {

// Device arrays of the fold order (Ctx: cut_kpos, cut_fpos, fold_K_slot /
// fold_K_ptr, fold_f_node / fold_f_ptr) from the context's class-ordered
// cut_nodes, cut_slot_ptr and cut_slot; node_enr flags the enrichment nodes.
int build_fold_device(Ctx& c, const std::vector<uint8_t>& node_enr, int n_entries) {
    cudaStream_t s = c.stream;
    DevScratch S(s);
    const int nc = c.n_cut;
    const long long nbk = c.n_blocks, nn = c.n_nodes;
    uint8_t *enr, *cutK, *cutF;
    int *cntK, *cntF, *fillK, *fillF, *tmpK, *tmpF, *runK, *runF;
    MESH_CUDA(S.alloc(&enr, nn));
    MESH_CUDA(S.alloc(&cutK, nbk));
    MESH_CUDA(S.alloc(&cutF, nn));
    MESH_CUDA(S.alloc(&cntK, nbk + 1));
    MESH_CUDA(S.alloc(&cntF, nn + 1));
    MESH_CUDA(S.alloc(&fillK, nbk));
    MESH_CUDA(S.alloc(&fillF, nn));
    MESH_CUDA(S.alloc(&tmpK, n_entries));
    MESH_CUDA(S.alloc(&tmpF, n_entries));
    MESH_CUDA(S.alloc(&runK, nbk));
    MESH_CUDA(S.alloc(&runF, nn));
    MESH_CUDA(cudaMemcpyAsync(enr, node_enr.data(), nn, cudaMemcpyHostToDevice, s));
    MESH_CUDA(cudaMemsetAsync(cutK, 0, nbk, s));
    MESH_CUDA(cudaMemcpyAsync(cutF, enr, nn, cudaMemcpyDeviceToDevice, s));
    MESH_CUDA(cudaMemsetAsync(cntK, 0, (nbk + 1) * sizeof(int), s));
    MESH_CUDA(cudaMemsetAsync(cntF, 0, (nn + 1) * sizeof(int), s));
    MESH_CUDA(cudaMemsetAsync(fillK, 0, nbk * sizeof(int), s));
    MESH_CUDA(cudaMemsetAsync(fillF, 0, nn * sizeof(int), s));
    k_fold_count<<<nb_mesh(nc), kThreadsMesh, 0, s>>>(nc, c.cut_slot_ptr, c.cut_slot, c.cut_nodes, enr, cntK, cutK,
                                                      cntF);
    int totK = 0, totF = 0, nrunK = 0, nrunF = 0;
    MESH_CUDA(exclusive_scan(S, cntK, nbk + 1, totK, s));
    MESH_CUDA(exclusive_scan(S, cntF, nn + 1, totF, s));
    k_fold_touched<<<nb_mesh(nbk), kThreadsMesh, 0, s>>>(nbk, cntK, runK);
    k_fold_touched<<<nb_mesh(nn), kThreadsMesh, 0, s>>>(nn, cntF, runF);
    MESH_CUDA(exclusive_scan(S, runK, nbk, nrunK, s));
    MESH_CUDA(exclusive_scan(S, runF, nn, nrunF, s));
    c.n_fold_K = nrunK;
    c.n_fold_f = nrunF;
    MESH_CUDA(cudaMalloc((void**)&c.fold_K_slot, std::max(1, nrunK) * sizeof(long long)));
    MESH_CUDA(cudaMalloc((void**)&c.fold_K_ptr, (nrunK + 1) * sizeof(int)));
    MESH_CUDA(cudaMalloc((void**)&c.fold_f_node, std::max(1, nrunF) * sizeof(int)));
    MESH_CUDA(cudaMalloc((void**)&c.fold_f_ptr, (nrunF + 1) * sizeof(int)));
    MESH_CUDA(cudaMalloc((void**)&c.cut_kpos, std::max(1, n_entries) * sizeof(int)));
    MESH_CUDA(cudaMalloc((void**)&c.cut_fpos, std::max(1, n_entries) * sizeof(int)));
    MESH_CUDA(cudaMemsetAsync(c.cut_kpos, 0xff, std::max(1, n_entries) * sizeof(int), s));
    MESH_CUDA(cudaMemsetAsync(c.cut_fpos, 0xff, std::max(1, n_entries) * sizeof(int), s));
    k_fold_runs<long long><<<nb_mesh(nbk), kThreadsMesh, 0, s>>>(nbk, cntK, runK, cutK, c.fold_K_slot, c.fold_K_ptr);
    k_fold_runs<int><<<nb_mesh(nn), kThreadsMesh, 0, s>>>(nn, cntF, runF, cutF, c.fold_f_node, c.fold_f_ptr);
    MESH_CUDA(cudaMemcpyAsync(c.fold_K_ptr + nrunK, &totK, sizeof(int), cudaMemcpyHostToDevice, s));
    MESH_CUDA(cudaMemcpyAsync(c.fold_f_ptr + nrunF, &totF, sizeof(int), cudaMemcpyHostToDevice, s));
    k_fold_scatter<<<nb_mesh(nc), kThreadsMesh, 0, s>>>(nc, c.cut_slot_ptr, c.cut_slot, c.cut_nodes, cntK, fillK,
                                                        tmpK, cntF, fillF, tmpF);
    k_fold_order<<<nb_mesh(nrunK), kThreadsMesh, 0, s>>>(nrunK, c.fold_K_ptr, tmpK, c.cut_kpos);
    k_fold_order<<<nb_mesh(nrunF), kThreadsMesh, 0, s>>>(nrunF, c.fold_f_ptr, tmpF, c.cut_fpos);
    // the runs of one contribution go straight into K; the rest stay with the fold
    int *multi, *midx;
    MESH_CUDA(S.alloc(&multi, std::max(1, nrunK)));
    MESH_CUDA(S.alloc(&midx, std::max(1, nrunK)));
    MESH_CUDA(cudaMalloc((void**)&c.cut_kdir, std::max(1, n_entries) * sizeof(long long)));
    MESH_CUDA(cudaMemsetAsync(c.cut_kdir, 0xff, std::max(1, n_entries) * sizeof(long long), s));
    k_fold_single<<<nb_mesh(nrunK), kThreadsMesh, 0, s>>>(nrunK, c.fold_K_ptr, tmpK, c.fold_K_slot, c.cut_kdir,
                                                          multi);
    k_fold_kdir_multi<<<nb_mesh(n_entries), kThreadsMesh, 0, s>>>(n_entries, c.cut_kpos, c.cut_kdir);
    int n_multi = 0;
    MESH_CUDA(cudaMemcpyAsync(midx, multi, std::max(1, nrunK) * sizeof(int), cudaMemcpyDeviceToDevice, s));
    MESH_CUDA(exclusive_scan(S, midx, nrunK, n_multi, s));
    c.n_fold_Km = n_multi;
    MESH_CUDA(cudaMalloc((void**)&c.fold_Km_slot, std::max(1, n_multi) * sizeof(long long)));
    MESH_CUDA(cudaMalloc((void**)&c.fold_Km_rng, std::max(1, n_multi) * sizeof(int2)));
    k_fold_multi<<<nb_mesh(nrunK), kThreadsMesh, 0, s>>>(nrunK, multi, midx, c.fold_K_slot, c.fold_K_ptr,
                                                         c.fold_Km_slot, c.fold_Km_rng);
    MESH_CUDA(cudaStreamSynchronize(s));
    MESH_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pgb

using namespace pgb;
