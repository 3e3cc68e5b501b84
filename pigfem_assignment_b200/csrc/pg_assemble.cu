// FP64 element integration and assembly kernels for sm_100a.
//
// Reference computation (PIGFEM 4.6.1):
//   Assembler::assemble_linear / assemble_elem_linear     src/Assembler.cpp:48-185
//   Assembler::assemble_nonlinear / assemble_elem_nonlinear src/Assembler.cpp:208-528
//   AssemblerLinearElasticity::KernelLinear               src/AssemblerLinearElasticity.cpp:24-38
//   AssemblerSmallStrainNonlinearStructural::Kernel*      src/AssemblerSmallStrainNonlinear.cpp:28-91
//   ProblemUtilities::SmallStrainKFast / Fast / IntForce  src/Utilities.cpp:196-408
//   ProblemUtilities::cohesiveDeltaFast / KFast / Force   src/Utilities.cpp:465-531
//   Mesh::store_shape_functions (recomputed, not cached)  src/Mesh.cpp:1443-1605
//   CohesiveElem::compute_rotation_general                src/CohesiveElem.cpp:207-238
//   OPCohesiveMaterial::Constitutive                      src/Material_OPCohesive.cpp:38-388
//
// Two kernels produce K (2x2-block CSR over nodes, FP64) and f_int:
//   k_assemble_tri: uncut triangles.  Per CTA slice of node rows, each
//     triangle's gradients are computed once per adjacent row into shared
//     memory, then one thread per 2x2 block (i, j) sums the constant-strain
//     B^T D B of the triangles joining i and j and stores it once with
//     coalesced 16-byte stores: no atomics, no prior clear.  Blocks of
//     enrichment rows and columns are written as zeros here.
//   k_assemble_cut: one warp per cut element.  Lanes own node-pair blocks of
//     the (3+n_enr)^2 element matrix, integrate every child (tri3/quad4/
//     polygon) and cohesive sub-element, and add into the rows with FP64
//     atomics (a few percent of elements).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>

#include "pg_internal.cuh"

namespace pgb {

__constant__ DevTemplate c_tmpl[32];
__constant__ DevChildQuad c_quad[kNumChildTypes];
// Global copies for reads whose address differs across a warp's lanes (the
// per-quadrature-point phase of the cut kernel): constant memory serialises
// those, the L1 serves them at once.
__device__ DevTemplate g_tmpl[32];
__device__ DevChildQuad g_quad[kNumChildTypes];

void upload_tables() {
    static bool done_dev[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done_dev[dev]) return;
    DevTemplate t[32] = {};
    const int nt = n_cut_templates();
    for (int i = 0; i < nt; ++i) {
        const CutTemplate& T = cut_template(i);
        t[i].n_enr = T.n_enr;
        t[i].n_child = T.n_child;
        t[i].n_coh = T.n_coh;
        for (int c = 0; c < T.n_child; ++c) {
            t[i].child_n[c] = T.child_n[c];
            t[i].child_type[c] = T.child_n[c] == 3 ? kChildTri3 : T.child_n[c] == 4 ? kChildQuad4
                                 : T.child_n[c] == 5 ? kChildPoly5 : kChildPoly6;
            for (int k = 0; k < T.child_n[c]; ++k) t[i].child_nodes[c][k] = T.child_nodes[c][k];
        }
        for (int c = 0; c < T.n_coh; ++c)
            for (int k = 0; k < 4; ++k) t[i].coh_nodes[c][k] = T.coh_nodes[c][k];
    }
    DevChildQuad q[kNumChildTypes] = {};
    for (int ty = 0; ty < kNumChildTypes; ++ty) {
        const ChildQuadrature& Q = child_quadrature(ty);
        q[ty].nq = Q.nq;
        q[ty].nn = Q.nn;
        for (int i = 0; i < Q.nq; ++i) q[ty].w[i] = Q.w[i];
        for (size_t i = 0; i < Q.N.size(); ++i) q[ty].N[i] = Q.N[i];
        for (size_t i = 0; i < Q.dN.size(); ++i) q[ty].dN[i] = Q.dN[i];
    }
    // A Tri3 child's shape gradients (and so its B^T D B) are the same at all
    // four points of its rule: the device integrates it at one point carrying
    // the summed weight, which equals the four-point sum up to rounding.
    {
        DevChildQuad& t3 = q[kChildTri3];
        double wsum = 0.0;
        for (int i = 0; i < t3.nq; ++i) wsum += t3.w[i];
        t3.nq = 1;
        t3.w[0] = wsum;
        const double third = 1.0 / 3.0;
        t3.N[0] = third;
        t3.N[1] = third;
        t3.N[2] = third;
    }
    cudaMemcpyToSymbol(c_tmpl, t, sizeof(t));
    cudaMemcpyToSymbol(c_quad, q, sizeof(q));
    cudaMemcpyToSymbol(g_tmpl, t, sizeof(t));
    cudaMemcpyToSymbol(g_quad, q, sizeof(q));
    if (dev >= 0 && dev < 64) done_dev[dev] = true;
}

// ---------------------------------------------------------------------------
// Uncut triangles: gather assembly, one thread per 2x2 block of K
// ---------------------------------------------------------------------------
constexpr int kTileMats = 32;                 // staged material table

void build_tri_map(const HostMesh& hm, int tile_nodes, std::vector<int>& map) {
    const int kTileNodes = tile_nodes, kTileEntries = 8 * tile_nodes;
    const int n = hm.n_nodes();
    map.assign((size_t)hm.n_blocks(), 0);
    for (int i = 0; i < n; ++i) {
        const int base = hm.ne_ptr[(i / kTileNodes) * kTileNodes];
        for (int q = hm.row_ptr[i]; q < hm.row_ptr[i + 1]; ++q) {
            const int j = hm.col[q];
            if (j == i) {
                map[q] = kTriMapDiag;
                continue;
            }
            int cnt = 0, word = 0;
            bool slow = false;
            for (int k = hm.ne_ptr[i]; k < hm.ne_ptr[i + 1]; ++k) {
                const int e = hm.ne_list[k] >> 2;
                int t = -1;
                for (int v = 0; v < 3; ++v)
                    if (hm.conn[3 * e + v] == j) t = v;
                if (t < 0) continue;
                const int rel = k - base;
                if (cnt >= 2 || rel >= kTileEntries) slow = true;
                else word |= (rel | (t << 10)) << (12 * cnt);
                ++cnt;
            }
            map[q] = slow ? kTriMapSlow : (word | (cnt << 24));
        }
    }
}

struct RowArgs {
    int n_nodes;
    int n_reg;
    const int* __restrict__ row_ptr;
    const int* __restrict__ col;
    const int* __restrict__ ne_ptr;
    const int* __restrict__ ne_list;
    const int* __restrict__ tri_map;
    const int* __restrict__ diag;
    const int4* __restrict__ elem4;
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ u;
    const double* __restrict__ dmat;
    int n_mat;
    double* K;
    double* f;
    int want_K, want_f;
};

// Block (v, t) of the constant-strain triangle e: B_v^T D B_t times the area
// (the reference's 4-point rule integrates the constant integrand exactly:
// its weights sum to 1/2, so K_e = J/2 * B^T D B with B = grad N / 1).
// Adds into k[4] when node j is a vertex of e.
__device__ __forceinline__ void cst_block_add(const RowArgs& a, int packed, int j, double k[4]) {
    const int e = packed >> 2, v = packed & 3;
    const int4 el = __ldg(&a.elem4[e]);
    const int t = el.x == j ? 0 : el.y == j ? 1 : el.z == j ? 2 : -1;
    if (t < 0) return;
    const double X0 = __ldg(&a.x[el.x]), X1 = __ldg(&a.x[el.y]), X2 = __ldg(&a.x[el.z]);
    const double Y0 = __ldg(&a.y[el.x]), Y1 = __ldg(&a.y[el.y]), Y2 = __ldg(&a.y[el.z]);
    const double J = (X1 - X0) * (Y2 - Y0) - (X2 - X0) * (Y1 - Y0);
    const double b0 = Y1 - Y2, b1 = Y2 - Y0, b2 = Y0 - Y1;
    const double c0 = X2 - X1, c1 = X0 - X2, c2 = X1 - X0;
    const double d11 = __ldg(&a.dmat[3 * el.w]), d12 = __ldg(&a.dmat[3 * el.w + 1]), d33 = __ldg(&a.dmat[3 * el.w + 2]);
    const double s = 0.5 / J;
    const double ba = (v == 0 ? b0 : v == 1 ? b1 : b2) * s;
    const double ca = (v == 0 ? c0 : v == 1 ? c1 : c2) * s;
    const double bb = t == 0 ? b0 : t == 1 ? b1 : b2;
    const double cb = t == 0 ? c0 : t == 1 ? c1 : c2;
    k[0] += ba * d11 * bb + ca * d33 * cb;
    k[1] += ba * d12 * cb + ca * d33 * bb;
    k[2] += ca * d12 * bb + ba * d33 * cb;
    k[3] += ca * d11 * cb + ba * d33 * bb;
}

// f_int contribution of the uncut triangle `packed` to its vertex v:
// sum_t K_e(v, t) u_t.
__device__ __forceinline__ void cst_force_add(const RowArgs& a, int packed, double& fx, double& fy) {
    const int e = packed >> 2, v = packed & 3;
    const int4 el = __ldg(&a.elem4[e]);
    const double X0 = __ldg(&a.x[el.x]), X1 = __ldg(&a.x[el.y]), X2 = __ldg(&a.x[el.z]);
    const double Y0 = __ldg(&a.y[el.x]), Y1 = __ldg(&a.y[el.y]), Y2 = __ldg(&a.y[el.z]);
    const double J = (X1 - X0) * (Y2 - Y0) - (X2 - X0) * (Y1 - Y0);
    const double b[3] = {Y1 - Y2, Y2 - Y0, Y0 - Y1};
    const double c[3] = {X2 - X1, X0 - X2, X1 - X0};
    const double d11 = __ldg(&a.dmat[3 * el.w]), d12 = __ldg(&a.dmat[3 * el.w + 1]), d33 = __ldg(&a.dmat[3 * el.w + 2]);
    const double s = 0.5 / J;
    const double ba = (v == 0 ? b[0] : v == 1 ? b[1] : b[2]) * s;
    const double ca = (v == 0 ? c[0] : v == 1 ? c[1] : c[2]) * s;
    const int nid[3] = {el.x, el.y, el.z};
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        const double bb = b[t], cb = c[t];
        const double ux = a.u[2 * nid[t]], uy = a.u[2 * nid[t] + 1];
        fx += (ba * d11 * bb + ca * d33 * cb) * ux + (ba * d12 * cb + ca * d33 * bb) * uy;
        fy += (ca * d12 * bb + ba * d33 * cb) * ux + (ca * d11 * cb + ba * d33 * bb) * uy;
    }
}

// Adds the staged triangle's block (own vertex, t) to k[4]: g = {b0, b1, b2,
// c0, c1, c2, 1/(2J)}, w = material | (own vertex << 16).
__device__ __forceinline__ void cst_staged_add(const double* g, int w, int t, const double* dm, double k[4]) {
    const int mat = w & 0xffff, v = w >> 16;
    const double s = g[6];
    const double ba = g[v] * s, ca = g[3 + v] * s, bb = g[t], cb = g[3 + t];
    const double d11 = dm[3 * mat], d12 = dm[3 * mat + 1], d33 = dm[3 * mat + 2];
    k[0] += ba * d11 * bb + ca * d33 * cb;
    k[1] += ba * d12 * cb + ca * d33 * bb;
    k[2] += ca * d12 * bb + ba * d33 * cb;
    k[3] += ca * d11 * cb + ba * d33 * bb;
}

// A CTA owns the 2x2-block CSR slice of kTileNodes consecutive node rows
// and works in three phases:
//   1. the slice's (node, adjacent uncut triangle) entries are gathered with
//      all of a thread's loads in flight together (entry, then triangle, then
//      coordinates), and each triangle's gradients b_t, c_t and 1/(2J) are
//      stored once per entry in shared memory, next to the slice's column
//      indices and the material table;
//   2. one thread per off-diagonal 2x2 block (i, j) of the slice finds the
//      (at most two) staged triangles of row i that contain node j and sums
//      their constant-strain blocks B_i^T D B_j (the reference's 4-point rule
//      integrates the constant integrand exactly: its weights sum to 1/2);
//      one thread per row sums the diagonal block over all the row's
//      triangles.  Keeping the two apart keeps the warps' FP64 work uniform
//      (two contributions per off-diagonal block).  Every block is stored once
//      with coalesced 16-byte stores: no atomics, no prior clear (blocks
//      coupling to enrichment nodes, and rows of enrichment nodes, are written
//      as zeros and completed by the cut-element kernel);
//   3. with WANT_F, one thread per row forms f_int,i = sum_e K_e(i, :) u_e
//      from the staged entries.
// A slice with more entries than the staging buffer (never for structured
// meshes, whose valence is at most 8) evaluates the blocks straight from
// global memory instead.
template <bool WANT_F, int TN>
__global__ void __launch_bounds__(2 * TN, 320 / TN) k_assemble_tri(RowArgs a, int n_tiles) {
    constexpr int kTileNodes = TN, kTileThreads = 2 * TN, kTileEntries = 8 * TN;
    constexpr int kEntriesPerThread = kTileEntries / kTileThreads;
    __shared__ double sG[kTileEntries][7];   // b0, b1, b2, c0, c1, c2, 1/(2J)
    __shared__ int4 sN[kTileEntries];        // n0, n1, n2, material | (entry's own vertex << 16)
    __shared__ double sD[3 * kTileMats];
    __shared__ int srp[kTileNodes + 1];
    __shared__ int sne[kTileNodes + 1];
    // a grid smaller than the tile count walks the tiles (persistent launch)
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int node0 = tile * kTileNodes;
    const int node_end = min(node0 + kTileNodes, a.n_nodes);
    const int nn = node_end - node0;
    // slice bounds read directly (broadcast loads), so that the entry and
    // column loads need not wait for the shared copies
    const int seg0 = __ldg(&a.row_ptr[node0]);
    const int nseg = __ldg(&a.row_ptr[node_end]) - seg0;
    const int k0 = __ldg(&a.ne_ptr[node0]);
    const int nent = __ldg(&a.ne_ptr[node_end]) - k0;
    const bool staged = nent <= kTileEntries;
    const bool mats_staged = a.n_mat <= kTileMats;
    for (int i = threadIdx.x; i <= nn; i += kTileThreads) {
        srp[i] = __ldg(&a.row_ptr[node0 + i]) - seg0;
        sne[i] = __ldg(&a.ne_ptr[node0 + i]) - k0;
    }
    if (mats_staged)
        for (int i = threadIdx.x; i < 3 * a.n_mat; i += kTileThreads) sD[i] = __ldg(&a.dmat[i]);
    if (staged) {
        int packed[kEntriesPerThread];
        int4 el[kEntriesPerThread];
#pragma unroll
        for (int u = 0; u < kEntriesPerThread; ++u) {
            const int k = threadIdx.x + u * kTileThreads;
            packed[u] = k < nent ? __ldg(&a.ne_list[k0 + k]) : 0;
        }
#pragma unroll
        for (int u = 0; u < kEntriesPerThread; ++u) {
            const int k = threadIdx.x + u * kTileThreads;
            el[u] = k < nent ? __ldg(&a.elem4[packed[u] >> 2]) : make_int4(0, 0, 0, 0);
        }
        double X[kEntriesPerThread][3], Y[kEntriesPerThread][3];
#pragma unroll
        for (int u = 0; u < kEntriesPerThread; ++u) {
            const int k = threadIdx.x + u * kTileThreads;
            if (k < nent) {
                X[u][0] = __ldg(&a.x[el[u].x]);
                X[u][1] = __ldg(&a.x[el[u].y]);
                X[u][2] = __ldg(&a.x[el[u].z]);
                Y[u][0] = __ldg(&a.y[el[u].x]);
                Y[u][1] = __ldg(&a.y[el[u].y]);
                Y[u][2] = __ldg(&a.y[el[u].z]);
            }
        }
#pragma unroll
        for (int u = 0; u < kEntriesPerThread; ++u) {
            const int k = threadIdx.x + u * kTileThreads;
            if (k < nent) {
                const double J = (X[u][1] - X[u][0]) * (Y[u][2] - Y[u][0]) - (X[u][2] - X[u][0]) * (Y[u][1] - Y[u][0]);
                double* g = sG[k];
                g[0] = Y[u][1] - Y[u][2];
                g[1] = Y[u][2] - Y[u][0];
                g[2] = Y[u][0] - Y[u][1];
                g[3] = X[u][2] - X[u][1];
                g[4] = X[u][0] - X[u][2];
                g[5] = X[u][1] - X[u][0];
                g[6] = 0.5 / J;
                sN[k] = make_int4(el[u].x, el[u].y, el[u].z, el[u].w | ((packed[u] & 3) << 16));
            }
        }
    }
    __syncthreads();
    for (int sidx = threadIdx.x; sidx < nseg; sidx += kTileThreads) {
        const int w = __ldg(&a.tri_map[seg0 + sidx]);
        if (staged && (w & kTriMapDiag)) continue;  // diagonal blocks: below
        double k[4] = {0.0, 0.0, 0.0, 0.0};
        if (staged && !(w & kTriMapSlow)) {
            // the (at most two) staged triangles joining the block's two nodes
            const int cnt = (w >> 24) & 3;
            if (cnt > 0) {
                const int e0 = w & 1023;
                cst_staged_add(sG[e0], sN[e0].w, (w >> 10) & 3, mats_staged ? sD : a.dmat, k);
            }
            if (cnt > 1) {
                const int e1 = (w >> 12) & 1023;
                cst_staged_add(sG[e1], sN[e1].w, (w >> 22) & 3, mats_staged ? sD : a.dmat, k);
            }
        } else {
            // row of this block: the largest li with srp[li] <= sidx
            int lo = 0, hi = nn - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (srp[mid] <= sidx) lo = mid; else hi = mid - 1;
            }
            const int j = __ldg(&a.col[seg0 + sidx]);
            for (int kk = k0 + sne[lo]; kk < k0 + sne[lo + 1]; ++kk) cst_block_add(a, __ldg(&a.ne_list[kk]), j, k);
        }
        if (a.want_K) {
            double2* dst = reinterpret_cast<double2*>(a.K + 4 * ((size_t)seg0 + sidx));
            dst[0] = make_double2(k[0], k[1]);
            dst[1] = make_double2(k[2], k[3]);
        }
    }
    if (staged) {
        // diagonal blocks: every triangle of the row contributes (t = own vertex)
        for (int li = threadIdx.x; li < nn; li += kTileThreads) {
            double k[4] = {0.0, 0.0, 0.0, 0.0};
            for (int kk = sne[li]; kk < sne[li + 1]; ++kk)
                cst_staged_add(sG[kk], sN[kk].w, sN[kk].w >> 16, mats_staged ? sD : a.dmat, k);
            if (a.want_K) {
                double2* dst = reinterpret_cast<double2*>(a.K + 4 * (size_t)__ldg(&a.diag[node0 + li]));
                dst[0] = make_double2(k[0], k[1]);
                dst[1] = make_double2(k[2], k[3]);
            }
        }
    }
    if (WANT_F) {
    // the cut-element kernel adds its own f_int contributions afterwards
    for (int li = threadIdx.x; li < nn; li += kTileThreads) {
        double fx = 0.0, fy = 0.0;
        if (staged) {
            for (int kk = sne[li]; kk < sne[li + 1]; ++kk) {
                const int4 el = sN[kk];
                const int mat = el.w & 0xffff, v = el.w >> 16;
                const double* g = sG[kk];
                const double s = g[6];
                const double ba = g[v] * s, ca = g[3 + v] * s;
                const double* D = mats_staged ? sD + 3 * mat : a.dmat + 3 * mat;
                const double d11 = D[0], d12 = D[1], d33 = D[2];
                const int nid[3] = {el.x, el.y, el.z};
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    const double bb = g[t], cb = g[3 + t];
                    const double ux = a.u[2 * nid[t]], uy = a.u[2 * nid[t] + 1];
                    fx += (ba * d11 * bb + ca * d33 * cb) * ux + (ba * d12 * cb + ca * d33 * bb) * uy;
                    fy += (ca * d12 * bb + ba * d33 * cb) * ux + (ca * d11 * cb + ba * d33 * bb) * uy;
                }
            }
        } else {
            for (int kk = k0 + sne[li]; kk < k0 + sne[li + 1]; ++kk) cst_force_add(a, __ldg(&a.ne_list[kk]), fx, fy);
        }
        a.f[2 * (node0 + li)] = fx;
        a.f[2 * (node0 + li) + 1] = fy;
    }
    }
    __syncthreads();  // the next tile reuses the shared buffers
    }
}

// ---------------------------------------------------------------------------
// Cohesive laws (FP64)
// ---------------------------------------------------------------------------
// delta = {tangential, normal} opening in the element's (t, n) frame; may be
// modified by the tiny-opening guard of OPCohesiveNUMaterial::getDeltaEff
// (Material_OPCohesiveNU.cpp:45-63).
__device__ void cohesive_law(const DevCohLaw& L, double dt, double dmax_c, double delta[2], double t[2],
                             double D[2][2], double& dmax_trial) {
    const double beta2 = (L.law == PG_COH_OP) ? L.p[2] * L.p[2] : L.p[3] * L.p[3];
    double d0 = delta[0], d1 = delta[1];
    if (d0 * d0 + d1 * d1 < 1e-40) { d0 = 1e-20; d1 = 1e-20; }
    delta[0] = d0;
    delta[1] = d1;
    if (L.law == PG_COH_OP) {
        const double sc = L.p[0], dc = L.p[1], visc = L.p[3];
        const double de = sqrt(d1 * d1 + beta2 * (d0 * d0));
        double T, dT;
        dmax_trial = dmax_c;
        if (de >= dmax_c || de < 0.0) {
            const double ex = exp(1.0 - de / dc);
            T = sc * (de / dc) * ex + visc / sc * (de - dmax_c) / dt / dc;
            dT = (sc / dc) * (1.0 - de / dc) * ex + visc / sc / dt / dc;
            dmax_trial = de;
        } else {
            const double Tm = sc * (dmax_c / dc) * exp(1.0 - dmax_c / dc);
            T = Tm * (de / dmax_c);
            dT = Tm / dmax_c;
        }
        const double br0 = beta2 * d0;
        const double br1 = beta2 * d1 + (1.0 - beta2) * d1;
        const double s = T / de;
        t[0] = s * br0;
        t[1] = s * br1;
        const double dd0 = beta2 * d0 / de, dd1 = d1 / de;
        const double aa = dT * de - T;
        const double de2 = de * de;
        D[0][0] = br0 * aa * (dd0 / de2) + s * beta2;
        D[0][1] = br0 * aa * (dd1 / de2);
        D[1][0] = br1 * aa * (dd0 / de2);
        D[1][1] = br1 * aa * (dd1 / de2) + s * (beta2 + (1.0 - beta2));
        return;
    }
    // bilinear penalty law with a compression penalty on the normal opening
    const double sc = L.p[0], Gc = L.p[1], Kp = L.p[2], eta = L.p[4];
    const double dlt0 = sc / Kp, dltf = 2.0 * Gc / sc;
    const double dn = d1 > 0.0 ? d1 : 0.0;
    const double de = sqrt(dn * dn + beta2 * (d0 * d0)) + 1e-300;
    auto env = [&](double dd, double& T, double& dT) {
        if (dd <= dlt0) { T = Kp * dd; dT = Kp; }
        else if (dd < dltf) { T = sc * (dltf - dd) / (dltf - dlt0); dT = -sc / (dltf - dlt0); }
        else { T = 0.0; dT = 0.0; }
    };
    double T, dT;
    dmax_trial = dmax_c;
    if (de >= dmax_c) {
        env(de, T, dT);
        // viscous regularisation while loading (eta = 0: none)
        T += eta * (de - dmax_c) / dt;
        dT += eta / dt;
        dmax_trial = de;
    } else {
        double Tm, dTm;
        env(dmax_c, Tm, dTm);
        T = Tm * (de / dmax_c);
        dT = Tm / dmax_c;
    }
    const double s = T / de;
    const double aa = dT * de - T;
    const double de2 = de * de;
    const double br0 = beta2 * d0, br1 = dn;
    const double dd0 = beta2 * d0 / de, dd1 = dn / de;
    t[0] = s * br0;
    D[0][0] = br0 * aa * (dd0 / de2) + s * beta2;
    if (d1 >= 0.0) {
        t[1] = s * br1;
        D[0][1] = br0 * aa * (dd1 / de2);
        D[1][0] = br1 * aa * (dd0 / de2);
        D[1][1] = br1 * aa * (dd1 / de2) + s;
    } else {
        t[1] = Kp * d1;
        D[0][1] = 0.0;
        D[1][0] = 0.0;
        D[1][1] = Kp;
    }
}

// ---------------------------------------------------------------------------
// Cut-element kernels
// ---------------------------------------------------------------------------

// Quadrature points of a child type on the device (a Tri3 child: one, see upload_tables)
int device_child_nq(int type) { return type == kChildTri3 ? 1 : child_quadrature(type).nq; }

int device_point_count(int tmpl) {
    const CutTemplate& T = cut_template(tmpl);
    int n = 0;
    for (int c = 0; c < T.n_child; ++c)
        n += device_child_nq(T.child_n[c] == 3 ? kChildTri3 : T.child_n[c] == 4 ? kChildQuad4
                             : T.child_n[c] == 5 ? kChildPoly5 : kChildPoly6);
    return n;
}

// One quadrature row: point q of a child with nc nodes (local numbers ln,
// coordinates cx, cy) of a cut element with nl local functions, material dm
// and parent (Tri3) gradients pbx, pby:
//   {w det, d11, d12, d33, (gx, gy) of each local function},
// value i at row[i * rs].
__device__ __forceinline__ void cut_row(double* row, int rs, int nl, const DevChildQuad& Q, int q, int nc,
                                        const int* ln, const double* cx, const double* cy, const double* dm,
                                        const double* pbx, const double* pby) {
    double J00 = 0.0, J01 = 0.0, J10 = 0.0, J11 = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxChildNodes; ++k) {
        if (k < nc) {
            const double dr = Q.dN[(q * nc + k) * 2], ds = Q.dN[(q * nc + k) * 2 + 1];
            J00 += dr * cx[k];
            J01 += dr * cy[k];
            J10 += ds * cx[k];
            J11 += ds * cy[k];
        }
    }
    const double det = J00 * J11 - J01 * J10;
    const double wgt = det * Q.w[q];
    // a zero weight (collapsed child) contributes nothing: the reference's
    // K_el.AXPY is cblas_daxpy, which returns at once for alpha == 0;
    // the row is zeroed so that no 0/0 gradient enters the sums
    const bool live = wgt != 0.0;
    row[0] = live ? wgt : 0.0;
    row[rs] = dm[0];
    row[2 * rs] = dm[1];
    row[3 * rs] = dm[2];
    for (int j = 0; j < 3; ++j) {
        row[(4 + 2 * j) * rs] = pbx[j];
        row[(5 + 2 * j) * rs] = pby[j];
    }
    for (int j = 3; j < nl; ++j) {
        row[(4 + 2 * j) * rs] = 0.0;
        row[(5 + 2 * j) * rs] = 0.0;
    }
    if (live) {
        const double idet = 1.0 / det;
#pragma unroll
        for (int k = 0; k < kMaxChildNodes; ++k) {
            if (k < nc && ln[k] >= 3) {
                const double dr = Q.dN[(q * nc + k) * 2], ds = Q.dN[(q * nc + k) * 2 + 1];
                row[(4 + 2 * ln[k]) * rs] = (J11 * dr - J01 * ds) * idet;
                row[(5 + 2 * ln[k]) * rs] = (-J10 * dr + J00 * ds) * idet;
            }
        }
    }
}

// parent (Tri3) gradients from the three parent coordinates
__device__ __forceinline__ void parent_gradients(const double* PX, const double* PY, double* pbx, double* pby) {
    const double PJ = (PX[1] - PX[0]) * (PY[2] - PY[0]) - (PX[2] - PX[0]) * (PY[1] - PY[0]);
    const double iPJ = 1.0 / PJ;  // one division per element instead of six
    pbx[0] = (PY[1] - PY[2]) * iPJ;
    pbx[1] = (PY[2] - PY[0]) * iPJ;
    pbx[2] = (PY[0] - PY[1]) * iPJ;
    pby[0] = (PX[2] - PX[1]) * iPJ;
    pby[1] = (PX[0] - PX[2]) * iPJ;
    pby[2] = (PX[1] - PX[0]) * iPJ;
}

// child ch and its point q holding point l of a template
__device__ __forceinline__ void point_child(const DevTemplate& TG, int l, int& ch, int& q) {
    ch = 0;
    q = l;
    while (q >= g_quad[TG.child_type[ch]].nq) {
        q -= g_quad[TG.child_type[ch]].nq;
        ++ch;
    }
}

// Quadrature row of one cut-element point.  What a point needs of the mesh
// is static, so the host packs it into one 64-byte record (kCutPointInts
// ints, see build_cut_points): the thread reads its record (cut_point_load),
// then the coordinates it names, and writes the row {w det, d11, d12, d33,
// (gx, gy) of each local function} contiguously (cut_point_row).
struct CutPoint {
    int4 r0, r1, r2, r3;
};

__device__ __forceinline__ CutPoint cut_point_load(const int4* __restrict__ rec) {
    return CutPoint{__ldg(rec), __ldg(rec + 1), __ldg(rec + 2), __ldg(rec + 3)};
}

__device__ __forceinline__ void cut_point_row(const CutPoint& P, const double* __restrict__ x,
                                              const double* __restrict__ y, const double* __restrict__ dmat,
                                              double* row) {
    const int gn[kMaxChildNodes] = {P.r0.x, P.r0.y, P.r0.z, P.r0.w, P.r1.x, P.r1.y};
    const int mat = P.r2.y, lnp = P.r2.z, meta = P.r2.w;
    const int q = meta & 255, type = (meta >> 8) & 3, nc = (meta >> 10) & 7, nl = (meta >> 13) & 15;
    int ln[kMaxChildNodes];
    double cx[kMaxChildNodes], cy[kMaxChildNodes];
#pragma unroll
    for (int k = 0; k < kMaxChildNodes; ++k) {
        ln[k] = (lnp >> (4 * k)) & 15;
        cx[k] = cy[k] = 0.0;
        if (k < nc) {
            cx[k] = __ldg(&x[gn[k]]);
            cy[k] = __ldg(&y[gn[k]]);
        }
    }
    const double PX[3] = {__ldg(&x[P.r1.z]), __ldg(&x[P.r1.w]), __ldg(&x[P.r2.x])};
    const double PY[3] = {__ldg(&y[P.r1.z]), __ldg(&y[P.r1.w]), __ldg(&y[P.r2.x])};
    double pbx[3], pby[3];
    parent_gradients(PX, PY, pbx, pby);
    const double dm[3] = {__ldg(&dmat[3 * mat]), __ldg(&dmat[3 * mat + 1]), __ldg(&dmat[3 * mat + 2])};
    cut_row(row, 1, nl, g_quad[type], q, nc, ln, cx, cy, dm, pbx, pby);
}

// Point records of the cut-element kernel, per point kCutPointInts ints:
// global nodes of its child (6, unused ones repeat the first), of the parent
// (3), the child's material, the child nodes' local numbers (4 bits each),
// then point q (8 bits), child type (2), child node count (3) and the
// element's local-function count (4), then the offset in doubles of the
// point's row (2 ints, low first: the element's first row + l (4 + 2 NL)),
// the element's point count and the point's number l within it.  Points are
// in class order, each element's in the order of its rows; one sentinel
// record follows the last point, holding only the rows' total length.
void build_cut_points(const std::vector<int>& nodes, const std::vector<int>& tmpl, const std::vector<int>& chm,
                      const std::vector<long long>& roff, const int* class_off, std::vector<int>& out,
                      std::vector<int>& pt_off) {
    // each element's records have a fixed place (the prefix of the points
    // before it), so the elements fill them in parallel
    const int nc = (int)tmpl.size();
    std::vector<long long> rec0(nc + 1, 0);
    std::vector<int> cls(nc, 0);
    for (int k = 0; k < kCutClasses; ++k)
        for (int oi = class_off[k]; oi < class_off[k + 1]; ++oi) cls[oi] = k;
    for (int oi = 0; oi < nc; ++oi) rec0[oi + 1] = rec0[oi] + device_point_count(tmpl[oi]);
    pt_off.assign(rec0.begin(), rec0.end());
    out.assign((size_t)(rec0[nc] + 1) * kCutPointInts, 0);
    parallel_for(nc, 2048, [&](long long oi) {
        const int k = cls[oi];
        const CutTemplate& T = cut_template(tmpl[oi]);
        const int* en = &nodes[(size_t)kCutNodeStride * oi];
        const int nq_e = device_point_count(tmpl[oi]);
        int* r = &out[(size_t)rec0[oi] * kCutPointInts];
        int l = 0;
        for (int ch = 0; ch < T.n_child; ++ch) {
            const int nc_ = T.child_n[ch];
            const int type = nc_ == 3 ? kChildTri3 : nc_ == 4 ? kChildQuad4 : nc_ == 5 ? kChildPoly5 : kChildPoly6;
            int lnp = 0;
            for (int c = 0; c < nc_; ++c) lnp |= T.child_nodes[ch][c] << (4 * c);
            for (int q = 0; q < device_child_nq(type); ++q, ++l, r += kCutPointInts) {
                for (int c = 0; c < kMaxChildNodes; ++c) r[c] = en[c < nc_ ? T.child_nodes[ch][c] : 0];
                r[6] = en[0];
                r[7] = en[1];
                r[8] = en[2];
                r[9] = chm[(size_t)kMaxChildren * oi + ch];
                r[10] = lnp;
                r[11] = q | (type << 8) | (nc_ << 10) | ((3 + T.n_enr) << 13);
                const long long off = roff[oi] + (long long)l * (4 + 2 * kCutClassNl[k]);
                r[12] = (int)(unsigned)(off & 0xffffffffLL);
                r[13] = (int)(off >> 32);
                r[14] = nq_e;
                r[15] = l;
            }
        }
    });
    // sentinel after the last point: its row offset is the rows' total length
    int* r = &out[(size_t)rec0[nc] * kCutPointInts];
    const long long total = roff.back();
    r[12] = (int)(unsigned)(total & 0xffffffffLL);
    r[13] = (int)(total >> 32);
}

void cut_row_spans(const std::vector<long long>& roff, const int* class_off, int span[4][3]) {
    for (int k = 0; k < kCutClasses; ++k)
        for (int w = 0; w < 3; ++w) {
            const int epc = cut_elems_per_cta(32 * kCutCtaWarps[w], kCutClassNl[k]);
            long long widest = 0;
            for (int e0 = class_off[k]; e0 < class_off[k + 1]; e0 += epc) {
                const int e1 = std::min(class_off[k + 1], e0 + epc);
                widest = std::max(widest, roff[e1] - roff[e0]);
            }
            span[k][w] = (int)std::min<long long>(widest, 1LL << 30);
        }
}

// ---------------------------------------------------------------------------
// Uncut triangles of a structured background grid: one thread per node row
// ---------------------------------------------------------------------------
// The background mesh is nx x ny cells of two triangles each (element
// 2 (i + j nx) + t, diagonal alternating with (i + j) % 2), regular node
// (i, j) = i + j (nx + 1).  Row (i, j) of K holds the node's grid neighbours
// -- all four axis neighbours, and the four diagonal ones for even nodes
// ((i + j) % 2 == 0), the only nodes a cell diagonal passes through -- in
// ascending order, then enrichment columns; grid_pattern_ok checks that
// layout on the host before this kernel is used.
//
// A CTA stages a tile's node coordinates (and displacements) with a
// one-node halo and the materials of its cells in shared memory -- coalesced
// loads, all in flight at once, one barrier -- and then a thread owns one
// regular node and writes its row: in registers, it forms row v of the
// constant-strain stiffness of every uncut triangle around the node (8 for
// an even node, 4 for an odd one; the reference's 4-point rule integrates
// the constant integrand exactly, its weights summing to 1/2), sums them
// into the node's grid-neighbour blocks and stores each block once with a
// 256-bit store.  A triangle is thus formed by each of its three vertices'
// threads; the FP64 pipe has room for that, and nothing but the inputs is
// staged or exchanged.  The lanes of a warp take nodes of one parity from
// one grid row (every other node column), so every lane runs the same,
// fully unrolled triangle code.
// Enrichment columns and enrichment rows are not touched: the cut-element
// fold writes them whole.  With WF the thread also forms its two f_int
// entries from the same row blocks.

// Corner (di + 2 dj) of local vertex m of triangle t in a cell of parity cp
// ((i + j) % 2): {n00, n10, n11}, {n00, n11, n01} for even cells,
// {n00, n10, n01}, {n10, n11, n01} for odd ones.
__host__ __device__ constexpr int tri_corner(int cp, int t, int m) {
    return cp == 0 ? (t == 0 ? (m == 0 ? 0 : m == 1 ? 1 : 3) : (m == 0 ? 0 : m == 1 ? 3 : 2))
                   : (t == 0 ? (m == 0 ? 0 : m == 1 ? 1 : 2) : (m == 0 ? 1 : m == 1 ? 3 : 2));
}

// Grid neighbours of node (gi, gj) present in its row, as bits d = 3 (dy + 1)
// + (dx + 1) (bit 4 the node itself): axis neighbours inside the grid, and
// the diagonal ones too for even nodes.  A block's place in the row is the
// number of lower bits set.
__host__ __device__ inline unsigned grid_nbr_mask(int gi, int gj, int nx, int ny) {
    const bool even = ((gi + gj) & 1) == 0;
    const bool w = gi > 0, e = gi < nx, s = gj > 0, n = gj < ny;
    return (s && even && w ? 1u : 0u) | (s ? 2u : 0u) | (s && even && e ? 4u : 0u) | (w ? 8u : 0u) | 16u |
           (e ? 32u : 0u) | (n && even && w ? 64u : 0u) | (n ? 128u : 0u) | (n && even && e ? 256u : 0u);
}

// Programmatic dependent launch (sm_90 and later).  A kernel launched with
// launch_pdl may start while the kernel before it on the stream is still
// running, once every CTA of that one has called pdl_trigger (or exited);
// pdl_wait blocks until the kernel before has completed and its writes are
// visible.  Both are no-ops for a kernel launched the ordinary way.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// One 2x2 block as a single 256-bit store (K is a cudaMalloc allocation, so
// every block is 32-byte aligned).
__device__ __forceinline__ void store_block(double* K, long long q, double k0, double k1, double k2, double k3) {
    double* dst = K + 4 * q;
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(dst), "d"(k0), "d"(k1), "d"(k2), "d"(k3) : "memory");
}

struct GridArgs {
    const int4* __restrict__ tiles;     // per CTA: grid block, I0, J0
    const int4* __restrict__ rves;      // per grid block: nx, ny, first node, first element
    const int* __restrict__ row_ptr;
    const int* __restrict__ emat;       // per element: material, -1 for cut elements
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ u;
    const double* __restrict__ dmat;
    double* K;
    double* f;
};

// Local vertex of the node in triangle T of the cell at offset (OX - 1,
// OY - 1) from a node of parity Q (the node is that cell's corner
// (1 - OX, 1 - OY)); -1 when the triangle does not contain it.
template <int Q, int OX, int OY, int T>
struct GridTri {
    static constexpr int cp = (Q + OX + OY) & 1;  // parity of the cell
    static constexpr int cn = (1 - OX) + 2 * (1 - OY);
    static constexpr int v = tri_corner(cp, T, 0) == cn ? 0 : tri_corner(cp, T, 1) == cn ? 1
                           : tri_corner(cp, T, 2) == cn ? 2 : -1;
    // position of vertex m in the node's 3 x 3 neighbourhood
    __host__ __device__ static constexpr int dx(int m) { return OX + (tri_corner(cp, T, m) & 1); }
    __host__ __device__ static constexpr int dy(int m) { return OY + (tri_corner(cp, T, m) >> 1); }
};

// The node's cell at offset (OX - 1, OY - 1), staged: corners (c & 1, c >> 1)
// of the cell as (x, y) pairs, and its two triangles' materials.
struct GridCell {
    double2 p[4];
    int m0, m1;
};

// 2 x (signed area) of triangle T of the cell
template <int Q, int OX, int OY, int T>
__device__ __forceinline__ double grid_tri_J(const GridCell& C) {
    using G = GridTri<Q, OX, OY, T>;
    const double2 P0 = C.p[tri_corner(G::cp, T, 0)], P1 = C.p[tri_corner(G::cp, T, 1)], P2 = C.p[tri_corner(G::cp, T, 2)];
    return (P1.x - P0.x) * (P2.y - P0.y) - (P2.x - P0.x) * (P1.y - P0.y);
}

// Adds row v (the node's) of triangle T's stiffness, scaled by s = 1 / (2 J),
// to the neighbour blocks acc[d] (d = 3 dy + dx; acc[4] = diagonal block as
// k00, k01, k11) and, with WF, K_vw u_w to (fx, fy); U: the cell's corner
// displacements.
template <int Q, int OX, int OY, int T, bool WK, bool WF>
__device__ __forceinline__ void grid_tri_row(const GridCell& C, const double2 (&U)[4], double s,
                                             const double* __restrict__ D, double (&acc)[9][4], double& fx,
                                             double& fy) {
    using G = GridTri<Q, OX, OY, T>;
    constexpr int v = G::v;
    const double2 P0 = C.p[tri_corner(G::cp, T, 0)], P1 = C.p[tri_corner(G::cp, T, 1)], P2 = C.p[tri_corner(G::cp, T, 2)];
    const double b[3] = {P1.y - P2.y, P2.y - P0.y, P0.y - P1.y};
    const double c[3] = {P2.x - P1.x, P0.x - P2.x, P1.x - P0.x};
    const double E0 = s * __ldg(&D[0]), E1 = s * __ldg(&D[1]), E2 = s * __ldg(&D[2]);
    const double bv = b[v], cv = c[v];
    const double Xv = bv * E0, Yv = bv * E1, Zv = bv * E2, Uv = cv * E0, Vv = cv * E1, Wv = cv * E2;
#pragma unroll
    for (int w = 0; w < 3; ++w) {
        const int d = 3 * G::dy(w) + G::dx(w);
        const double k0 = Xv * b[w] + Wv * c[w];
        const double k1 = Yv * c[w] + Wv * b[w];
        const double k2 = Vv * b[w] + Zv * c[w];
        const double k3 = Uv * c[w] + Zv * b[w];
        if (WK) {
            if (w == v) {
                acc[4][0] += k0;
                acc[4][1] += k1;
                acc[4][2] += k3;
            } else {
                acc[d][0] += k0;
                acc[d][1] += k1;
                acc[d][2] += k2;
                acc[d][3] += k3;
            }
        }
        if (WF) {
            const double2 uw = U[tri_corner(G::cp, T, w)];
            fx += k0 * uw.x + k1 * uw.y;
            fy += k2 * uw.x + k3 * uw.y;
        }
    }
}

// The uncut triangles of cell (OX, OY) around the node (materials -1 for
// cut or absent triangles).  When both contain the node, their two scales
// share one division.
template <int Q, int OX, int OY, bool WK, bool WF>
__device__ __forceinline__ void grid_cell(const GridCell& C, const double2 (&U)[4], const double* __restrict__ dmat,
                                          double (&acc)[9][4], double& fx, double& fy) {
    constexpr bool h0 = GridTri<Q, OX, OY, 0>::v >= 0, h1 = GridTri<Q, OX, OY, 1>::v >= 0;
    if constexpr (h0 && h1) {
        if (C.m0 < 0 && C.m1 < 0) return;
        const double J0 = grid_tri_J<Q, OX, OY, 0>(C), J1 = grid_tri_J<Q, OX, OY, 1>(C);
        const double r = 0.5 / (J0 * J1);
        if (C.m0 >= 0) grid_tri_row<Q, OX, OY, 0, WK, WF>(C, U, r * J1, dmat + 3 * C.m0, acc, fx, fy);
        if (C.m1 >= 0) grid_tri_row<Q, OX, OY, 1, WK, WF>(C, U, r * J0, dmat + 3 * C.m1, acc, fx, fy);
    } else if constexpr (h0) {
        if (C.m0 < 0) return;
        grid_tri_row<Q, OX, OY, 0, WK, WF>(C, U, 0.5 / grid_tri_J<Q, OX, OY, 0>(C), dmat + 3 * C.m0, acc, fx, fy);
    } else {
        if (C.m1 < 0) return;
        grid_tri_row<Q, OX, OY, 1, WK, WF>(C, U, 0.5 / grid_tri_J<Q, OX, OY, 1>(C), dmat + 3 * C.m1, acc, fx, fy);
    }
}

template <int D>
__device__ __forceinline__ void grid_store(double* K, int q0, unsigned mask, const double (&acc)[9][4]) {
    if (mask & (1u << D)) {
        const long long q = q0 + __popc(mask & ((1u << D) - 1u));
        if (D == 4) store_block(K, q, acc[4][0], acc[4][1], acc[4][1], acc[4][2]);
        else store_block(K, q, acc[D][0], acc[D][1], acc[D][2], acc[D][3]);
    }
}

// Tile of the structured-grid kernel: kGridTileC node columns (I0 even) x
// TR node rows (2 or 4, picked by the autotuner), one thread per node; warp
// 2 r + q takes the nodes of parity q in tile row r (every other column).
// Staged window: the tile's nodes with a one-node halo, the cells around them.
constexpr int kGridTileC = kGridTileCols;
constexpr int kGridWinX = kGridTileC + 2;   // staged node columns
constexpr int kGridCellX = kGridTileC + 1;  // staged cell columns

template <int OX, int OY, bool WF>
__device__ __forceinline__ void grid_load_cell(GridCell& C, double2 (&U)[4], const double2* sXY, const double2* sU,
                                               const int2* sM, int lx, int ly) {
    // cell (OX, OY) of the node at window position (lx, ly): its corner (cx, cy)
    // is window node (lx - 1 + OX + cx, ly - 1 + OY + cy)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int w = (ly - 1 + OY + (k >> 1)) * kGridWinX + lx - 1 + OX + (k & 1);
        C.p[k] = sXY[w];
        if (WF) U[k] = sU[w];
    }
    const int2 m = sM[(ly - 1 + OY) * kGridCellX + lx - 1 + OX];
    C.m0 = m.x;
    C.m1 = m.y;
}

template <int Q, bool WK, bool WF>
__device__ __forceinline__ void grid_node(const GridArgs& a, const int4 B, int gi, int gj, int lx, int ly,
                                          const double2* sXY, const double2* sU, const int2* sM) {
    const int node = B.z + gi + gj * (B.x + 1);
    const int q0 = WK ? __ldg(&a.row_ptr[node]) : 0;
    const unsigned mask = grid_nbr_mask(gi, gj, B.x, B.y);
    double acc[9][4];
#pragma unroll
    for (int d = 0; d < 9; ++d) acc[d][0] = acc[d][1] = acc[d][2] = acc[d][3] = 0.0;
    double fx = 0.0, fy = 0.0;
    GridCell C;
    double2 U[4];
    // cells in the order that completes blocks early: below (d = 0, 1, 2
    // done), above left (d = 3, 6), above right (d = 4, 5, 7, 8)
    grid_load_cell<0, 0, WF>(C, U, sXY, sU, sM, lx, ly);
    grid_cell<Q, 0, 0, WK, WF>(C, U, a.dmat, acc, fx, fy);
    grid_load_cell<1, 0, WF>(C, U, sXY, sU, sM, lx, ly);
    grid_cell<Q, 1, 0, WK, WF>(C, U, a.dmat, acc, fx, fy);
    if (WK) {
        if (Q == 0) grid_store<0>(a.K, q0, mask, acc);
        grid_store<1>(a.K, q0, mask, acc);
        if (Q == 0) grid_store<2>(a.K, q0, mask, acc);
    }
    grid_load_cell<0, 1, WF>(C, U, sXY, sU, sM, lx, ly);
    grid_cell<Q, 0, 1, WK, WF>(C, U, a.dmat, acc, fx, fy);
    if (WK) {
        grid_store<3>(a.K, q0, mask, acc);
        if (Q == 0) grid_store<6>(a.K, q0, mask, acc);
    }
    grid_load_cell<1, 1, WF>(C, U, sXY, sU, sM, lx, ly);
    grid_cell<Q, 1, 1, WK, WF>(C, U, a.dmat, acc, fx, fy);
    if (WK) {
        grid_store<4>(a.K, q0, mask, acc);
        grid_store<5>(a.K, q0, mask, acc);
        grid_store<7>(a.K, q0, mask, acc);
        if (Q == 0) grid_store<8>(a.K, q0, mask, acc);
    }
    if (WF) {
        a.f[2 * (size_t)node] = fx;
        a.f[2 * (size_t)node + 1] = fy;
    }
}

// One CTA per tile: the window's coordinates (and displacements) and cell
// materials are staged with coalesced loads, all in flight together; then
// every thread forms its node's row from shared memory.
template <bool WK, bool WF, int TR>
__global__ void __launch_bounds__(kGridTileC * TR, 12 / TR) k_grid_rows(GridArgs a) {
    pdl_trigger();  // the cut elements' row kernels may fill the SMs this grid frees
    constexpr int kGridThreads = kGridTileC * TR, kGridWinY = TR + 2, kGridCellY = TR + 1;
    __shared__ double2 sXY[kGridWinX * kGridWinY];
    __shared__ double2 sU[WF ? kGridWinX * kGridWinY : 1];
    __shared__ int2 sM[kGridCellX * kGridCellY];
    const int4 T = __ldg(&a.tiles[blockIdx.x]);
    const int4 B = __ldg(&a.rves[T.x]);  // this tile's grid block: nx, ny, first node, first element
    const int nx = B.x, ny = B.y, NX1 = nx + 1;
    const int I0 = T.y, J0 = T.z;
    for (int i = threadIdx.x; i < kGridWinX * kGridWinY; i += kGridThreads) {
        const int gi = I0 - 1 + i % kGridWinX, gj = J0 - 1 + i / kGridWinX;
        double2 v = make_double2(0.0, 0.0), uv = make_double2(0.0, 0.0);
        if (gi >= 0 && gi <= nx && gj >= 0 && gj <= ny) {
            const size_t n = (size_t)B.z + gi + (size_t)gj * NX1;
            v = make_double2(__ldg(&a.x[n]), __ldg(&a.y[n]));
            if (WF) uv = make_double2(__ldg(&a.u[2 * n]), __ldg(&a.u[2 * n + 1]));
        }
        sXY[i] = v;
        if (WF) sU[i] = uv;
    }
    for (int i = threadIdx.x; i < kGridCellX * kGridCellY; i += kGridThreads) {
        const int ci = I0 - 1 + i % kGridCellX, cj = J0 - 1 + i / kGridCellX;
        sM[i] = (ci >= 0 && ci < nx && cj >= 0 && cj < ny)
                    ? __ldg(reinterpret_cast<const int2*>(a.emat) + ((size_t)B.w / 2 + ci + (size_t)cj * nx))
                    : make_int2(-1, -1);
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = w >> 1, q = w & 1;
    const int gj = J0 + r;
    const int gi = I0 + 2 * lane + ((gj + q) & 1);
    if (gj > ny || gi > nx) return;  // no barrier follows
    const int lx = gi - I0 + 1, ly = r + 1;
    if (q == 0) grid_node<0, WK, WF>(a, B, gi, gj, lx, ly, sXY, sU, sM);
    else grid_node<1, WK, WF>(a, B, gi, gj, lx, ly, sXY, sU, sM);
}

// Asynchronous copies into shared memory (cp.async, Ampere and later): an
// 8-byte copy, zero-filled when `valid` is false (the source address is then
// only a placeholder and is not read: src-size 0).
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The staged window of one tile (k_grid_rows_pipe): coordinates as (x, y)
// pairs, displacements, cell materials.
template <int TR, bool WF>
struct GridWin {
    double2 xy[kGridWinX * (TR + 2)];
    double2 u[WF ? kGridWinX * (TR + 2) : 1];
    int2 m[kGridCellX * (TR + 1)];
};

// Issues the copies of tile t's window into W (every thread its share).
template <int TR, bool WF>
__device__ __forceinline__ void grid_stage_async(const GridArgs& a, int t, GridWin<TR, WF>& W) {
    constexpr int kThreads = kGridTileC * TR, kWinY = TR + 2, kCellY = TR + 1;
    const int4 T = __ldg(&a.tiles[t]);
    const int4 B = __ldg(&a.rves[T.x]);
    const int nx = B.x, ny = B.y, NX1 = nx + 1;
    for (int i = threadIdx.x; i < kGridWinX * kWinY; i += kThreads) {
        const int gi = T.y - 1 + i % kGridWinX, gj = T.z - 1 + i / kGridWinX;
        const bool in = gi >= 0 && gi <= nx && gj >= 0 && gj <= ny;
        const size_t n = in ? (size_t)B.z + gi + (size_t)gj * NX1 : 0;
        cp_async8(&W.xy[i].x, a.x + n, in);
        cp_async8(&W.xy[i].y, a.y + n, in);
        if (WF) {
            cp_async8(&W.u[i].x, a.u + 2 * n, in);
            cp_async8(&W.u[i].y, a.u + 2 * n + 1, in);
        }
    }
    for (int i = threadIdx.x; i < kGridCellX * kCellY; i += kThreads) {
        const int ci = T.y - 1 + i % kGridCellX, cj = T.z - 1 + i / kGridCellX;
        const bool in = ci >= 0 && ci < nx && cj >= 0 && cj < ny;
        const size_t k = in ? (size_t)B.w / 2 + ci + (size_t)cj * nx : 0;
        cp_async8(&W.m[i], reinterpret_cast<const int2*>(a.emat) + k, in);
    }
}

// Persistent variant of k_grid_rows: each CTA walks the tile table with a
// stride of the grid, and copies the next tile's window into a free one of
// three shared-memory buffers (cp.async) while its threads form the rows of
// the current one, so that the staging latency overlaps the arithmetic
// instead of idling the SM.  With three buffers one barrier per tile
// suffices: the buffer refilled in iteration k was last read in iteration
// k - 2, which every thread has left once it passed iteration k - 1's
// barrier.  Out-of-grid window entries are zero-filled (materials:
// out-of-grid cells read as material 0 from the fill, so they are set to -1
// after the copy lands).
template <bool WK, bool WF, int TR>
__global__ void __launch_bounds__(kGridTileC * TR, 12 / TR) k_grid_rows_pipe(GridArgs a, int n_tiles) {
    pdl_trigger();
    __shared__ GridWin<TR, WF> W[3];
    int t = blockIdx.x;
    if (t >= n_tiles) return;
    grid_stage_async<TR, WF>(a, t, W[0]);
    cp_async_commit();
    for (int k = 0; t < n_tiles; t += gridDim.x, ++k) {
        GridWin<TR, WF>& cur = W[k % 3];
        const int tn = t + gridDim.x;
        if (tn < n_tiles) grid_stage_async<TR, WF>(a, tn, W[(k + 1) % 3]);
        cp_async_commit();  // (an empty group when nothing was issued)
        cp_async_wait_one();  // the current tile's copies have landed
        const int4 T = __ldg(&a.tiles[t]);
        const int4 B = __ldg(&a.rves[T.x]);
        const int nx = B.x, ny = B.y;
        // cells outside the grid are no triangles
        for (int i = threadIdx.x; i < kGridCellX * (TR + 1); i += kGridTileC * TR) {
            const int ci = T.y - 1 + i % kGridCellX, cj = T.z - 1 + i / kGridCellX;
            if (!(ci >= 0 && ci < nx && cj >= 0 && cj < ny)) cur.m[i] = make_int2(-1, -1);
        }
        __syncthreads();
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int r = w >> 1, q = w & 1;
        const int gj = T.z + r;
        const int gi = T.y + 2 * lane + ((gj + q) & 1);
        if (gj <= ny && gi <= nx) {
            const int lx = gi - T.y + 1, ly = r + 1;
            if (q == 0) grid_node<0, WK, WF>(a, B, gi, gj, lx, ly, cur.xy, cur.u, cur.m);
            else grid_node<1, WK, WF>(a, B, gi, gj, lx, ly, cur.xy, cur.u, cur.m);
        }
    }
    cp_async_wait_all();
}

// True when every regular row of the block pattern is laid out as
// k_grid_rows assumes: the node's grid neighbours (grid_nbr_mask) and
// itself in ascending order, then only enrichment columns; checked per grid
// block (one per RVE of a batch).
static bool grid_block_pattern_ok(const HostMesh& hm, const HostMesh::GridBlock& gb) {
    const int nx = gb.nx, ny = gb.ny, no = gb.node_off;
    if ((long long)(nx + 1) * (ny + 1) != gb.n_reg || gb.elem_off % 2) return false;
    for (int gj = 0; gj <= ny; ++gj)
        for (int gi = 0; gi <= nx; ++gi) {
            const int i = no + gi + gj * (nx + 1);
            const unsigned mask = grid_nbr_mask(gi, gj, nx, ny);
            int q = hm.row_ptr[i];
            for (int d = 0; d < 9; ++d) {
                if (!(mask & (1u << d))) continue;
                const int j = no + (gi + d % 3 - 1) + (gj + d / 3 - 1) * (nx + 1);
                if (q >= hm.row_ptr[i + 1] || hm.col[q] != j) return false;
                ++q;
            }
            // then only this block's enrichment nodes
            for (; q < hm.row_ptr[i + 1]; ++q)
                if (hm.col[q] < no + gb.n_reg) return false;
        }
    // the block's elements are its grid cells in order
    for (int e = 0; e < 2 * nx * ny; e += 2 * nx) {
        const int ge = gb.elem_off + e;
        const int cj = e / (2 * nx);
        if (hm.conn[3 * (size_t)ge] != no + cj * (nx + 1)) return false;
    }
    return true;
}

bool grid_pattern_ok(const HostMesh& hm) {
    if (hm.grids.empty()) return false;
    // every grid block, in parallel
    std::atomic<bool> ok{true};
    parallel_for((long long)hm.grids.size(), 1, [&](long long g) {
        if (ok.load(std::memory_order_relaxed) && !grid_block_pattern_ok(hm, hm.grids[g])) ok.store(false);
    });
    return ok.load();
}

void launch_grid(const Ctx& c, const double* U, bool want_f, bool want_K, cudaStream_t s) {
    GridArgs ga;
    ga.rves = c.grid_rves;
    ga.row_ptr = c.row_ptr;
    ga.emat = c.grid_emat;
    ga.x = c.x;
    ga.y = c.y;
    ga.u = U;
    ga.dmat = c.dmat;
    ga.K = c.K;
    ga.f = c.F;
    const int tr = c.tuning.grid_block == 128 ? 2 : 4;  // threads per CTA = 64 x node rows per tile
    ga.tiles = c.grid_tiles[tr == 2 ? 0 : 1];
    const int blocks = c.n_grid_tiles[tr == 2 ? 0 : 1];
    if (blocks == 0) return;
    if (c.tuning.tri_persistent) {
        // persistent, pipelined: as many CTAs as fit on the SMs at once
        int dev = 0, n_sm = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        auto go = [&](auto kern) {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kGridTileC * tr, 0);
            if (c.tuning.cut_overlap > 0 && c.n_cut > 0) per_sm -= c.tuning.cut_overlap;  // room for the cut kernels
            const int grid = std::min(blocks, std::max(1, per_sm) * n_sm);
            kern<<<grid, kGridTileC * tr, 0, s>>>(ga, blocks);
        };
        if (tr == 2) {
            if (want_K && want_f) go(k_grid_rows_pipe<true, true, 2>);
            else if (want_K) go(k_grid_rows_pipe<true, false, 2>);
            else if (want_f) go(k_grid_rows_pipe<false, true, 2>);
        } else {
            if (want_K && want_f) go(k_grid_rows_pipe<true, true, 4>);
            else if (want_K) go(k_grid_rows_pipe<true, false, 4>);
            else if (want_f) go(k_grid_rows_pipe<false, true, 4>);
        }
        return;
    }
    if (tr == 2) {
        if (want_K && want_f) k_grid_rows<true, true, 2><<<blocks, kGridTileC * 2, 0, s>>>(ga);
        else if (want_K) k_grid_rows<true, false, 2><<<blocks, kGridTileC * 2, 0, s>>>(ga);
        else if (want_f) k_grid_rows<false, true, 2><<<blocks, kGridTileC * 2, 0, s>>>(ga);
    } else {
        if (want_K && want_f) k_grid_rows<true, true, 4><<<blocks, kGridTileC * 4, 0, s>>>(ga);
        else if (want_K) k_grid_rows<true, false, 4><<<blocks, kGridTileC * 4, 0, s>>>(ga);
        else if (want_f) k_grid_rows<false, true, 4><<<blocks, kGridTileC * 4, 0, s>>>(ga);
    }
}

// ---------------------------------------------------------------------------
// Cut elements: integration per element row, then a fold of shared slots
// ---------------------------------------------------------------------------
// Every cut element's (3 + n_enr)^2 node-pair blocks have a fixed place in
// the element's slot table (cut_slot: pair (a, b) at cut_slot_ptr + a nl +
// b, holding the block's K slot).  k_cut_elems forms the element's
// quadrature rows in shared memory and integrates one row of blocks (a, *)
// per thread.  A block whose K slot takes no other contribution (half of
// them) goes into K there: stored where only cut elements reach the slot
// (enrichment rows and columns), else added to the triangle kernel's value
// by a reduction that waits for nothing -- with a single addend its result
// is the same in any order.  The others are stored at their position in
// fold order (kpos, built once per mesh: all contributions to one K slot
// next to each other, by element and pair), and for residual passes K_ab
// u_b at its position in the node-sorted order (fpos).  k_fold_K then gives
// every K slot of two or more contributions its final value in one thread:
// the triangle kernel's value (or zero, for blocks in enrichment rows or
// columns, which only cut elements reach) plus its contiguous run of
// contributions; k_fold_f does the same per node for f_int.  The sums are
// the same on every run.
//
// After the triangle kernel on the same stream, chained by programmatic
// dependent launch: k_coh_points forms every cohesive Gauss point (one
// thread each: traction-separation law, trial delta_max, row), k_cut_elems
// (one launch per size class) the quadrature rows and the blocks, then the
// folds.  k_cut_points forms the same quadrature rows in global memory for
// the stress recovery.
constexpr int kCohRow = kCohRowDoubles;  // {w dA, N0, N1, (R^T D R) 4, (R^T t) 2, pad}

// One thread per quadrature point: its row, point-major (the element's point
// l at row_off[element] + l (4 + 2 NL), NL its size class's largest local
// node count), so that a pair thread reads a point's values with four
// 128-bit loads.  The record carries the row's offset.  A CTA's points are
// consecutive, so their rows are one contiguous span: the threads form them
// in shared memory and the CTA stores the span with coalesced 128-bit stores.
constexpr int kPointThreads = 128;
constexpr int kRowMax = 4 + 2 * kCutClassNl[kCutClasses - 1];  // widest row (34 doubles)

__global__ void __launch_bounds__(kPointThreads) k_cut_points(int n_pts, const int4* __restrict__ pts,
                                                              const double* __restrict__ x,
                                                              const double* __restrict__ y,
                                                              const double* __restrict__ dmat, double* rows) {
    __shared__ __align__(16) double sRow[kPointThreads * kRowMax];
    pdl_trigger();  // reads only the mesh: runs beside the triangle kernel's last CTAs
    const int p0 = blockIdx.x * kPointThreads, p = p0 + threadIdx.x;
    const int p1 = min(n_pts, p0 + kPointThreads);
    // the CTA's span of rows: from its first point's row to the next CTA's
    // (the record after the last point is a sentinel holding the rows' end)
    const int4 rb = __ldg(pts + 4 * (size_t)p0 + 3), re = __ldg(pts + 4 * (size_t)p1 + 3);
    const long long base = (long long)(unsigned)rb.x | ((long long)rb.y << 32);
    const long long end = (long long)(unsigned)re.x | ((long long)re.y << 32);
    if (p < n_pts) {
        const CutPoint cp = cut_point_load(pts + 4 * (size_t)p);
        const long long off = (long long)(unsigned)cp.r3.x | ((long long)cp.r3.y << 32);
        cut_point_row(cp, x, y, dmat, sRow + (off - base));
    }
    __syncthreads();
    // rows hold an even number of doubles and start at even offsets
    const int n2 = (int)((end - base) / 2);
    const double2* src = reinterpret_cast<const double2*>(sRow);
    double2* dst = reinterpret_cast<double2*>(rows + base);
    for (int i = threadIdx.x; i < n2; i += kPointThreads) dst[i] = src[i];
    pdl_wait();  // completes only after the kernel before it: the chain stays ordered
}

// One thread per cohesive Gauss point (CohEdge2, 2 points, w = 1): the law
// at its opening (writing the trial delta_max) and its row.  Point qp of
// sub-element ce of element ci (class order) is qp = cut_coh_qp0[ci] + 2 ce
// + q; coh_rec[qp] packs ci << 8 | ce << 1 | q.
struct CohArgs {
    int n_qp;
    const int* __restrict__ coh_rec;
    const int* __restrict__ cut_nodes;
    const int* __restrict__ cut_tmpl;
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ u;
    const double* __restrict__ isv_c;
    double* isv_t;
    double* coh_rows;
    DevCohLaw coh;
    double dt;
};

__global__ void __launch_bounds__(128) k_coh_points(CohArgs a) {
    pdl_trigger();
    const int qp = blockIdx.x * blockDim.x + threadIdx.x;
    if (qp >= a.n_qp) {
        pdl_wait();
        return;
    }
    const int rec = __ldg(&a.coh_rec[qp]);
    const int ci = rec >> 8, ce = (rec >> 1) & 127, q = rec & 1;
    const DevTemplate& T = g_tmpl[__ldg(&a.cut_tmpl[ci])];
    const int* en = a.cut_nodes + (size_t)kCutNodeStride * ci;
    int n[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) n[m] = __ldg(&en[T.coh_nodes[ce][m]]);
    const double jx = 0.5 * (__ldg(&a.x[n[1]]) - __ldg(&a.x[n[0]]));
    const double jy = 0.5 * (__ldg(&a.y[n[1]]) - __ldg(&a.y[n[0]]));
    const double mag = sqrt(jx * jx + jy * jy);
    const double nx = -jy, ny = jx;
    const double dA = sqrt(nx * nx + ny * ny);
    const double R[2][2] = {{jx / mag, jy / mag}, {nx / dA, ny / dA}};
    const double xi = q == 0 ? -0.57735026918962576450914878050196 : 0.57735026918962576450914878050196;
    const double N0 = 0.5 * (1.0 - xi), N1 = 0.5 * (1 + xi);
    double dg[2];
#pragma unroll
    for (int d = 0; d < 2; ++d)
        dg[d] = N0 * (__ldg(&a.u[2 * n[2] + d]) - __ldg(&a.u[2 * n[0] + d])) +
                N1 * (__ldg(&a.u[2 * n[3] + d]) - __ldg(&a.u[2 * n[1] + d]));
    double dl[2] = {R[0][0] * dg[0] + R[0][1] * dg[1], R[1][0] * dg[0] + R[1][1] * dg[1]};
    double tr[2], Dc[2][2], dmax_t;
    cohesive_law(a.coh, a.dt, __ldg(&a.isv_c[qp]), dl, tr, Dc, dmax_t);
    a.isv_t[qp] = dmax_t;
    double* row = a.coh_rows + (size_t)kCohRow * qp;
    row[0] = dA * 1.0;
    row[1] = N0;
    row[2] = N1;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            double sum = 0.0;
#pragma unroll
            for (int k1 = 0; k1 < 2; ++k1)
#pragma unroll
                for (int k2 = 0; k2 < 2; ++k2) sum += R[k1][i] * Dc[k1][k2] * R[k2][j];
            row[3 + 2 * i + j] = sum;
        }
    row[7] = R[0][0] * tr[0] + R[1][0] * tr[1];
    row[8] = R[0][1] * tr[0] + R[1][1] * tr[1];
    row[9] = 0.0;
    pdl_wait();
}

struct ElemArgs {
    int n_elem;                     // elements of this size class
    int first;                      // its first element in class order
    const int* __restrict__ cut_nodes;
    const int* __restrict__ cut_tmpl;
    const int* __restrict__ cut_coh_qp0;
    const int* __restrict__ cut_slot_ptr;
    const int* __restrict__ kpos;   // slot-table entry -> position in fold order (-1: no K slot)
    const long long* __restrict__ kdir;  // slot-table entry -> slot << 1 | cut_only of a one-entry run,
                                         // else -2 - (fold position), -1 without a K slot (direct passes)
    const int* __restrict__ fpos;   // slot-table entry -> position in node order
    const int4* __restrict__ pts;   // point records (build_cut_points)
    const int* __restrict__ pt_off; // per element its first point record
    const long long* __restrict__ row_off;
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ dmat;
    const double* __restrict__ coh_rows;
    const double* __restrict__ u;
    double* ke;                     // 4 FP64 per fold position
    double* fe;                     // 2 FP64 per node-order position
    double* K;
    int want_K, want_f;
    int direct;                     // 1: one-entry runs go straight into K (the triangle kernel has finished)
};

__device__ __forceinline__ double2 lds2(const double* p) { return *reinterpret_cast<const double2*>(p); }

// One CTA per cut_elems_per_cta(blockDim.x, NL) consecutive elements of size
// class NL.  The CTA first forms its elements' quadrature rows in shared
// memory (one thread per point, from the point records; the mesh is all it
// reads, so this part runs beside the kernel before it), then one thread per
// local function a of an element integrates the element's row a of blocks:
// K_ab = sum_q w_q B_a^T D B_b over the rows for every b, plus the cohesive
// sub-elements' N_a N_b (+-) R^T D R terms where both nodes are cohesive
// nodes.  Residual passes store K_ab u_b (bulk) for every b and, on the
// diagonal block, add the node's cohesive traction term.  In direct passes
// a block whose K slot no other contribution reaches goes straight into K
// (stored, or added to the triangle kernel's value by a single-addend
// reduction); every other block goes to its place in fold order.
template <int NL, bool WF, bool COH>
__global__ void __launch_bounds__(256, NL <= 5 ? 3 : (NL <= 7 ? 2 : 1)) k_cut_elems(ElemArgs a) {
    extern __shared__ __align__(16) double sRow[];
    pdl_trigger();
    constexpr int W = 4 + 2 * NL;
    const int epc = cut_elems_per_cta(blockDim.x, NL);
    const int e0 = blockIdx.x * epc, e1 = min(a.n_elem, e0 + epc);
    const int c0 = a.first + e0;
    const long long base = __ldg(&a.row_off[c0]);
    // this thread's element and local function; its static tables are
    // loaded while the rows are formed
    const int le = threadIdx.x / NL, pa = threadIdx.x - le * NL;
    const bool act = le < epc && e0 + le < a.n_elem;
    const int ci = c0 + (act ? le : 0);
    const int tm = __ldg(&a.cut_tmpl[ci]);
    const long long r0 = __ldg(&a.row_off[ci]), r1 = __ldg(&a.row_off[ci + 1]);
    const int sp_e = __ldg(&a.cut_slot_ptr[ci]);
    {
        const int p0 = __ldg(&a.pt_off[c0]), p1 = __ldg(&a.pt_off[a.first + e1]);
        for (int p = p0 + (int)threadIdx.x; p < p1; p += blockDim.x) {
            const CutPoint cp = cut_point_load(a.pts + 4 * (size_t)p);
            const long long off = (long long)(unsigned)cp.r3.x | ((long long)cp.r3.y << 32);
            cut_point_row(cp, a.x, a.y, a.dmat, sRow + (off - base));
        }
    }
    __syncthreads();
    if (!act) return;
    const DevTemplate& T = g_tmpl[tm];
    const int nl = 3 + T.n_enr;
    if (pa >= nl) return;
    const int nq = (int)((r1 - r0) / W);
    const long long sp0 = sp_e + (long long)pa * nl;
    const int* en = a.cut_nodes + (size_t)kCutNodeStride * ci;
    // where the row's blocks go (static tables), in flight during the
    // integration: kdir in direct mode, else the fold position
    long long kd[NL];
#pragma unroll
    for (int b = 0; b < NL; ++b) {
        kd[b] = -1;
        if (a.want_K && b < nl) kd[b] = a.direct ? __ldg(&a.kdir[sp0 + b]) : -2 - (long long)__ldg(&a.kpos[sp0 + b]);
    }
    pdl_wait();  // the kernel before has finished: K's triangle values, the cohesive rows
    double k[NL][4];
#pragma unroll
    for (int b = 0; b < NL; ++b) k[b][0] = k[b][1] = k[b][2] = k[b][3] = 0.0;
    const double* rw = sRow + (r0 - base);
    for (int q = 0; q < nq; ++q, rw += W) {
        const double2 wd = lds2(rw), dd = lds2(rw + 2), ga = lds2(rw + 4 + 2 * pa);
        const double wgt = wd.x, d11 = wd.y, d12 = dd.x, d33 = dd.y;
        const double ba = ga.x * wgt, ca = ga.y * wgt;
#pragma unroll
        for (int b = 0; b < NL; ++b) {
            if (b < nl) {
                const double2 gb = lds2(rw + 4 + 2 * b);
                const double bb = gb.x, cb = gb.y;
                k[b][0] += ba * d11 * bb + ca * d33 * cb;
                k[b][1] += ba * d12 * cb + ca * d33 * bb;
                k[b][2] += ca * d12 * bb + ba * d33 * cb;
                k[b][3] += ca * d11 * cb + ba * d33 * bb;
            }
        }
    }
    // bulk internal force terms K_ab u_b (the cohesive part of f_int is the
    // traction integral below, not the cohesive tangent times u); every
    // block but the diagonal one is final here
    double fx = 0.0, fy = 0.0;
    if (WF) {
#pragma unroll
        for (int b = 0; b < NL; ++b) {
            if (b < nl) {
                const int nb = __ldg(&en[b]);
                const double ux = __ldg(&a.u[2 * nb]), uy = __ldg(&a.u[2 * nb + 1]);
                const double gx = k[b][0] * ux + k[b][1] * uy, gy = k[b][2] * ux + k[b][3] * uy;
                if (b == pa) {
                    fx = gx;
                    fy = gy;
                } else {
                    const int fp = __ldg(&a.fpos[sp0 + b]);
                    if (fp >= 0) reinterpret_cast<double2*>(a.fe)[fp] = make_double2(gx, gy);
                }
            }
        }
    }
    if (COH && T.n_coh > 0) {
        const int qp0 = __ldg(&a.cut_coh_qp0[ci]);
        for (int ce = 0; ce < T.n_coh; ++ce) {
            int i = -1;
#pragma unroll
            for (int m = 0; m < 4; ++m)
                if (T.coh_nodes[ce][m] == pa) i = m;
            if (i < 0) continue;
            const double sa = i < 2 ? -1.0 : 1.0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const double* row = a.coh_rows + (size_t)kCohRow * (qp0 + 2 * ce + q);
                const double wgt = __ldg(&row[0]);
                if (wgt == 0.0) continue;
                const double Na = __ldg(&row[1 + (i & 1)]);
                const double D0 = __ldg(&row[3]), D1 = __ldg(&row[4]), D2 = __ldg(&row[5]), D3 = __ldg(&row[6]);
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int b = T.coh_nodes[ce][m];
                    const double sgn = ((i < 2) == (m < 2)) ? 1.0 : -1.0;
                    const double v = wgt * sgn * Na * __ldg(&row[1 + (m & 1)]);
#pragma unroll
                    for (int bb = 0; bb < NL; ++bb)
                        if (bb == b) {
                            k[bb][0] += v * D0;
                            k[bb][1] += v * D1;
                            k[bb][2] += v * D2;
                            k[bb][3] += v * D3;
                        }
                }
                fx += wgt * sa * Na * __ldg(&row[7]);
                fy += wgt * sa * Na * __ldg(&row[8]);
            }
        }
    }
    if (WF) {
        const int fp = __ldg(&a.fpos[sp0 + pa]);
        if (fp >= 0) reinterpret_cast<double2*>(a.fe)[fp] = make_double2(fx, fy);
    }
    // kd >= 0: the slot's only contribution (slot << 1 | cut_only): stored
    // (a block only cut elements reach) or added to the triangle kernel's
    // value -- one addend, so the reduction is exact in any order and waits
    // for nothing; kd <= -2: the fold position -2 - kd
    if (a.want_K) {
#pragma unroll
        for (int b = 0; b < NL; ++b) {
            if (b < nl) {
                const long long v = kd[b];
                if (v >= 0) {
                    double* dst = a.K + 4 * (v >> 1);
                    if (v & 1) {
                        store_block(a.K, v >> 1, k[b][0], k[b][1], k[b][2], k[b][3]);
                    } else {
                        atomicAdd(dst, k[b][0]);
                        atomicAdd(dst + 1, k[b][1]);
                        atomicAdd(dst + 2, k[b][2]);
                        atomicAdd(dst + 3, k[b][3]);
                    }
                } else if (v <= -2) {
                    store_block(a.ke, -2 - v, k[b][0], k[b][1], k[b][2], k[b][3]);
                }
            }
        }
    }
}

// K slots that cut elements touch, one thread per run: K[slot] = (the
// triangle kernel's value, or 0 where flagged cut_only) + the slot's
// contiguous run of blocks ke[i0 .. i1), summed in run order.  fold_slot[j]
// = slot << 1 | cut_only; the run's range is rng[j] when given (the runs of
// two or more blocks, when k_cut_elems stored the others in K itself), else
// ptr[j] .. ptr[j + 1] (every run).
__global__ void __launch_bounds__(256) k_fold_K(int n, const long long* __restrict__ fold_slot,
                                                const int* __restrict__ fold_ptr, const int2* __restrict__ rng,
                                                const double* __restrict__ ke, double* K) {
    pdl_wait();  // the blocks, and (through the chain) the triangle kernel's K
    pdl_trigger();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const long long sw = __ldg(&fold_slot[j]);
    int i0, i1;
    if (rng) {
        const int2 r = __ldg(&rng[j]);
        i0 = r.x;
        i1 = r.y;
    } else {
        i0 = __ldg(&fold_ptr[j]);
        i1 = __ldg(&fold_ptr[j + 1]);
    }
    const long long slot = sw >> 1;
    // plain loads, so that the run's loads are all in flight at once
    double2 a01 = make_double2(0.0, 0.0), a23 = make_double2(0.0, 0.0);
    if (!(sw & 1)) {
        const double2* kb = reinterpret_cast<const double2*>(K + 4 * slot);
        a01 = kb[0];
        a23 = kb[1];
    }
    const double2* kv = reinterpret_cast<const double2*>(ke);
    for (int i = i0; i < i1; ++i) {
        const double2 v01 = __ldg(kv + 2 * (size_t)i), v23 = __ldg(kv + 2 * (size_t)i + 1);
        a01.x += v01.x;
        a01.y += v01.y;
        a23.x += v23.x;
        a23.y += v23.y;
    }
    store_block(K, slot, a01.x, a01.y, a23.x, a23.y);
}

// f_int of the nodes cut elements touch, one thread each: f = (the triangle
// kernel's value, or 0 for enrichment nodes) + the node's contiguous run of
// pair terms.  fold_node[j] = node << 1 | cut_only.
__global__ void __launch_bounds__(256) k_fold_f(int n, const int* __restrict__ fold_node,
                                                const int* __restrict__ fold_ptr, const double* __restrict__ fe,
                                                double* f) {
    pdl_wait();
    pdl_trigger();
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int nw = __ldg(&fold_node[j]);
    const int i0 = __ldg(&fold_ptr[j]), i1 = __ldg(&fold_ptr[j + 1]);
    const int node = nw >> 1;
    double2 acc = (nw & 1) ? make_double2(0.0, 0.0) : reinterpret_cast<const double2*>(f)[node];
    for (int i = i0; i < i1; ++i) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(fe) + i);
        acc.x += v.x;
        acc.y += v.y;
    }
    reinterpret_cast<double2*>(f)[node] = acc;
}

// Shape sensitivity of the cut elements' internal force (pg_sens.cu): one
// warp per cut element.  The element's enrichment nodes on the selected
// inclusion move by sgn * h_rel * r * (their velocity), the lanes form the
// element's quadrature rows at the moved geometry (one point per lane) in
// per-warp shared memory, integrate their node-pair blocks over them and
// dot the element's internal force (bulk K_e u_e plus the cohesive
// tractions) with wsens; lane 0 adds sgn * (that) / (2 h) to sens[inclusion].
// NL is the size class's largest local node count; PPL = ceil(NL^2 / 32)
// node-pair blocks per lane.
constexpr int kQpChunk = 32;

template <int NL, int PPL, int W>
__global__ void __launch_bounds__(32 * W, (NL <= 5 ? 24 : (NL <= 7 ? 16 : 8)) / W) k_cut_sens(CutArgs a) {
    constexpr int kQRow = 4 + 2 * NL;
    __shared__ double sX[W][NL], sY[W][NL];
    __shared__ double sU[W][2 * NL];
    __shared__ int sL[W][NL];
    __shared__ double sQ[W][kQpChunk][kQRow];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int oi = blockIdx.x * W + w;
    if (oi >= a.n_cut) return;
    const int ci = a.first + oi;  // class-ordered element index
    const int node = lane < NL ? __ldg(&a.cut_nodes[kCutNodeStride * ci + lane]) : -1;
    const int tmpl = __ldg(&a.cut_tmpl[ci]);
    const DevTemplate& T = c_tmpl[tmpl];
    const int nl = 3 + T.n_enr;
    if (lane < nl) {
        sL[w][lane] = node;
        sX[w][lane] = a.x[node];
        sY[w][lane] = a.y[node];
        sU[w][2 * lane] = a.u[2 * node];
        sU[w][2 * lane + 1] = a.u[2 * node + 1];
    }
    __syncwarp();
    const unsigned full = 0xffffffffu;
    const int my_inc = (lane >= 3 && lane < nl) ? a.node_inc[sL[w][lane]] : -1;
    // the which-th distinct inclusion among the enrichment slots, in slot order
    int sel = -1, count = 0;
    for (int l = 3; l < nl; ++l) {
        const int v = __shfl_sync(full, my_inc, l);
        bool seen = false;
        for (int l2 = 3; l2 < l; ++l2) seen |= __shfl_sync(full, my_inc, l2) == v;
        if (!seen && v >= 0) {
            if (count == a.which) sel = v;
            ++count;
        }
    }
    if (sel < 0) return;  // warp-uniform: no such inclusion in this element
    const double hstep = a.h_rel * a.radius[sel];
    if (lane < nl && my_inc == sel) {
        const int nd = sL[w][lane];
        sX[w][lane] += a.sgn * hstep * a.vel[2 * nd];
        sY[w][lane] += a.sgn * hstep * a.vel[2 * nd + 1];
    }
    __syncwarp();
    // parent (Tri3) gradients are constant over the element (its nodes have moved)
    double pbx[3], pby[3];
    parent_gradients(sX[w], sY[w], pbx, pby);
    int nq_total = 0;
    for (int ch = 0; ch < T.n_child; ++ch) nq_total += c_quad[T.child_type[ch]].nq;
    double acc[PPL][4];
#pragma unroll
    for (int k = 0; k < PPL; ++k) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0;
    const int npairs = nl * nl;
    int pa[PPL], pb[PPL];
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        const int p = lane + 32 * k;
        pa[k] = p / nl;
        pb[k] = p - pa[k] * nl;
    }
    for (int qbase = 0; qbase < nq_total; qbase += kQpChunk) {
        // geometry of one quadrature point per lane, all points in parallel
        const int l = qbase + lane;
        if (l < nq_total) {
            const DevTemplate& TG = g_tmpl[tmpl];
            int ch, q;
            point_child(TG, l, ch, q);
            const int nc = TG.child_n[ch];
            const int mat = a.cut_child_mat[ci * kMaxChildren + ch];
            int ln[kMaxChildNodes];
            double cx[kMaxChildNodes], cy[kMaxChildNodes];
#pragma unroll
            for (int k = 0; k < kMaxChildNodes; ++k) {
                ln[k] = k < nc ? TG.child_nodes[ch][k] : 0;
                cx[k] = sX[w][ln[k]];
                cy[k] = sY[w][ln[k]];
            }
            const double dm[3] = {a.dmat[3 * mat], a.dmat[3 * mat + 1], a.dmat[3 * mat + 2]};
            cut_row(sQ[w][lane], 1, nl, g_quad[TG.child_type[ch]], q, nc, ln, cx, cy, dm, pbx, pby);
        }
        __syncwarp();
        // each lane integrates its node-pair blocks over the chunk's points
        const int nqc = min(kQpChunk, nq_total - qbase);
        for (int q = 0; q < nqc; ++q) {
            const double* row = sQ[w][q];
            const double wgt = row[0], d11 = row[1], d12 = row[2], d33 = row[3];
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                if (lane + 32 * k < npairs) {
                    const double ba = row[4 + 2 * pa[k]] * wgt, ca = row[5 + 2 * pa[k]] * wgt;
                    const double bb = row[4 + 2 * pb[k]], cb = row[5 + 2 * pb[k]];
                    acc[k][0] += ba * d11 * bb + ca * d33 * cb;
                    acc[k][1] += ba * d12 * cb + ca * d33 * bb;
                    acc[k][2] += ca * d12 * bb + ba * d33 * cb;
                    acc[k][3] += ca * d11 * cb + ba * d33 * bb;
                }
            }
        }
        __syncwarp();
    }
    // this lane's share of wsens . f_e: bulk K_ab u_b ...
    double part = 0.0;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        if (lane + 32 * k < npairs) {
            const int ia = pa[k], ib = pb[k];
            const double ux = sU[w][2 * ib], uy = sU[w][2 * ib + 1];
            const double fx = acc[k][0] * ux + acc[k][1] * uy;
            const double fy = acc[k][2] * ux + acc[k][3] * uy;
            part += a.wsens[2 * sL[w][ia]] * fx + a.wsens[2 * sL[w][ia] + 1] * fy;
        }
    }
    // ... and the cohesive tractions: two Gauss points per sub-element, one lane each
    if (lane < 2 * T.n_coh) {
        const int ce = lane >> 1, q = lane & 1;
        const int c0 = T.coh_nodes[ce][0], c1 = T.coh_nodes[ce][1], c2 = T.coh_nodes[ce][2], c3 = T.coh_nodes[ce][3];
        const double jx = 0.5 * (sX[w][c1] - sX[w][c0]);
        const double jy = 0.5 * (sY[w][c1] - sY[w][c0]);
        const double mag = sqrt(jx * jx + jy * jy);
        const double nx = -jy, ny = jx;
        const double dA = sqrt(nx * nx + ny * ny);
        const double R[2][2] = {{jx / mag, jy / mag}, {nx / dA, ny / dA}};
        const double xi = q == 0 ? -0.57735026918962576450914878050196 : 0.57735026918962576450914878050196;
        const double N0 = 0.5 * (1.0 - xi), N1 = 0.5 * (1 + xi);
        double dg[2];
        for (int d = 0; d < 2; ++d)
            dg[d] = N0 * (sU[w][2 * c2 + d] - sU[w][2 * c0 + d]) + N1 * (sU[w][2 * c3 + d] - sU[w][2 * c1 + d]);
        double dl[2] = {R[0][0] * dg[0] + R[0][1] * dg[1], R[1][0] * dg[0] + R[1][1] * dg[1]};
        const int qp = a.cut_coh_qp0[ci] + lane;
        double tr[2], Dc[2][2], dmax_t;
        cohesive_law(a.coh, a.dt, a.isv_c[qp], dl, tr, Dc, dmax_t);
        const double tR0 = R[0][0] * tr[0] + R[1][0] * tr[1];
        const double tR1 = R[0][1] * tr[0] + R[1][1] * tr[1];
        const double wgt = dA * 1.0;
        if (wgt != 0.0) {
            const int cn[4] = {c0, c1, c2, c3};
            const double Nn[2] = {N0, N1};
            for (int m = 0; m < 4; ++m) {
                const double sgn = m < 2 ? -1.0 : 1.0;
                const int nd = sL[w][cn[m]];
                part += a.wsens[2 * nd] * (wgt * sgn * Nn[m & 1] * tR0) +
                        a.wsens[2 * nd + 1] * (wgt * sgn * Nn[m & 1] * tR1);
            }
        }
    }
    // central difference of wsens . f_e: this pass adds sgn * (its share) / (2 h)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(full, part, o);
    if (lane == 0) atomicAdd(&a.sens[sel], a.sgn * part / (2.0 * hstep));
}

// ---------------------------------------------------------------------------
// Analytic shape derivative of the cut elements' internal force
// (SensitivityShapeParameterStructural::KernelVolumetric,
// src/SensitivityShapeParameterStructural.cpp:18-90, and the cohesive
// traction's), by forward-mode differentiation: every coordinate carries its
// derivative along the parameter's velocity field (nonzero at the enrichment
// nodes of the parameter's inclusion), and the quadrature rows carry the
// derivatives of the weight w det J and of the enrichment gradients.  The
// derivative of sum_q w det J B^T D B u is then
//   sum_q [ d(w det J) B^T D B u + w det J (dB^T D B u + B^T D dB u) ],
// the reference's B^T (D dB u + sigma div v) + dB^T sigma weighted by w det J,
// exact to rounding (no step size).
struct Dual {
    double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double r = sqrt(a.v);
    return {r, 0.5 * a.d / r};
}

// cut_row with coordinates (cx, cy) moving at (dcx, dcy): the row's values
// and their derivatives; the parent gradients do not move (parent nodes have
// no velocity)
__device__ __forceinline__ void cut_row_dual(double* row, double* drow, int nl, const DevChildQuad& Q, int q, int nc,
                                             const int* ln, const double* cx, const double* cy, const double* dcx,
                                             const double* dcy, const double* dm, const double* pbx,
                                             const double* pby) {
    Dual J00{0.0, 0.0}, J01{0.0, 0.0}, J10{0.0, 0.0}, J11{0.0, 0.0};
#pragma unroll
    for (int k = 0; k < kMaxChildNodes; ++k) {
        if (k < nc) {
            const double dr = Q.dN[(q * nc + k) * 2], ds = Q.dN[(q * nc + k) * 2 + 1];
            const Dual X{cx[k], dcx[k]}, Y{cy[k], dcy[k]};
            J00 = J00 + dr * X;
            J01 = J01 + dr * Y;
            J10 = J10 + ds * X;
            J11 = J11 + ds * Y;
        }
    }
    const Dual det = J00 * J11 - J01 * J10;
    const Dual wgt = Q.w[q] * det;
    const bool live = wgt.v != 0.0;
    row[0] = live ? wgt.v : 0.0;
    drow[0] = live ? wgt.d : 0.0;
    for (int i = 1; i < 4; ++i) {
        row[i] = dm[i - 1];
        drow[i] = 0.0;
    }
    for (int j = 0; j < 3; ++j) {
        row[4 + 2 * j] = pbx[j];
        row[5 + 2 * j] = pby[j];
        drow[4 + 2 * j] = drow[5 + 2 * j] = 0.0;
    }
    for (int j = 3; j < nl; ++j) row[4 + 2 * j] = row[5 + 2 * j] = drow[4 + 2 * j] = drow[5 + 2 * j] = 0.0;
    if (live) {
#pragma unroll
        for (int k = 0; k < kMaxChildNodes; ++k) {
            if (k < nc && ln[k] >= 3) {
                const double dr = Q.dN[(q * nc + k) * 2], ds = Q.dN[(q * nc + k) * 2 + 1];
                const Dual gx = (dr * J11 - ds * J01) / det;
                const Dual gy = (ds * J00 - dr * J10) / det;
                row[4 + 2 * ln[k]] = gx.v;
                row[5 + 2 * ln[k]] = gy.v;
                drow[4 + 2 * ln[k]] = gx.d;
                drow[5 + 2 * ln[k]] = gy.d;
            }
        }
    }
}

// One warp per cut element and pass (which-th inclusion among its enrichment
// slots, one parameter kind): the derivative of wsens . f_e along the
// velocity field vel, added to sens[param_of[3 inclusion + kind]].
template <int NL, int PPL, int W>
__global__ void __launch_bounds__(32 * W) k_cut_sens_ad(CutArgs a) {
    constexpr int kQRow = 4 + 2 * NL;
    __shared__ double sX[W][NL], sY[W][NL], sDX[W][NL], sDY[W][NL];
    __shared__ double sU[W][2 * NL];
    __shared__ int sL[W][NL];
    __shared__ double sQ[W][kQpChunk][kQRow];
    __shared__ double sQd[W][kQpChunk][kQRow];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int oi = blockIdx.x * W + w;
    if (oi >= a.n_cut) return;
    const int ci = a.first + oi;
    const int node = lane < NL ? __ldg(&a.cut_nodes[kCutNodeStride * ci + lane]) : -1;
    const int tmpl = __ldg(&a.cut_tmpl[ci]);
    const DevTemplate& T = c_tmpl[tmpl];
    const int nl = 3 + T.n_enr;
    if (lane < nl) {
        sL[w][lane] = node;
        sX[w][lane] = a.x[node];
        sY[w][lane] = a.y[node];
        sU[w][2 * lane] = a.u[2 * node];
        sU[w][2 * lane + 1] = a.u[2 * node + 1];
    }
    __syncwarp();
    const unsigned full = 0xffffffffu;
    const int my_inc = (lane >= 3 && lane < nl) ? a.node_inc[sL[w][lane]] : -1;
    int sel = -1, count = 0;
    for (int l = 3; l < nl; ++l) {
        const int v = __shfl_sync(full, my_inc, l);
        bool seen = false;
        for (int l2 = 3; l2 < l; ++l2) seen |= __shfl_sync(full, my_inc, l2) == v;
        if (!seen && v >= 0) {
            if (count == a.which) sel = v;
            ++count;
        }
    }
    if (sel < 0) return;  // warp-uniform
    const int param = a.param_of[3 * sel + a.kind];
    if (param < 0) return;
    if (lane < nl) {
        const bool moves = my_inc == sel;
        const int nd = sL[w][lane];
        sDX[w][lane] = moves ? a.vel[2 * nd] : 0.0;
        sDY[w][lane] = moves ? a.vel[2 * nd + 1] : 0.0;
    }
    __syncwarp();
    double pbx[3], pby[3];
    parent_gradients(sX[w], sY[w], pbx, pby);
    int nq_total = 0;
    for (int ch = 0; ch < T.n_child; ++ch) nq_total += c_quad[T.child_type[ch]].nq;
    double acc[PPL][4];
#pragma unroll
    for (int k = 0; k < PPL; ++k) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0;
    const int npairs = nl * nl;
    int pa[PPL], pb[PPL];
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        const int p = lane + 32 * k;
        pa[k] = p / nl;
        pb[k] = p - pa[k] * nl;
    }
    for (int qbase = 0; qbase < nq_total; qbase += kQpChunk) {
        const int l = qbase + lane;
        if (l < nq_total) {
            const DevTemplate& TG = g_tmpl[tmpl];
            int ch, q;
            point_child(TG, l, ch, q);
            const int nc = TG.child_n[ch];
            const int mat = a.cut_child_mat[ci * kMaxChildren + ch];
            int ln[kMaxChildNodes];
            double cx[kMaxChildNodes], cy[kMaxChildNodes], dcx[kMaxChildNodes], dcy[kMaxChildNodes];
#pragma unroll
            for (int k = 0; k < kMaxChildNodes; ++k) {
                ln[k] = k < nc ? TG.child_nodes[ch][k] : 0;
                cx[k] = sX[w][ln[k]];
                cy[k] = sY[w][ln[k]];
                dcx[k] = sDX[w][ln[k]];
                dcy[k] = sDY[w][ln[k]];
            }
            const double dm[3] = {a.dmat[3 * mat], a.dmat[3 * mat + 1], a.dmat[3 * mat + 2]};
            cut_row_dual(sQ[w][lane], sQd[w][lane], nl, g_quad[TG.child_type[ch]], q, nc, ln, cx, cy, dcx, dcy, dm,
                         pbx, pby);
        }
        __syncwarp();
        const int nqc = min(kQpChunk, nq_total - qbase);
        for (int q = 0; q < nqc; ++q) {
            const double* row = sQ[w][q];
            const double* drow = sQd[w][q];
            const double wgt = row[0], dwgt = drow[0], d11 = row[1], d12 = row[2], d33 = row[3];
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                if (lane + 32 * k < npairs) {
                    const double ba = row[4 + 2 * pa[k]], ca = row[5 + 2 * pa[k]];
                    const double bb = row[4 + 2 * pb[k]], cb = row[5 + 2 * pb[k]];
                    const double dba = drow[4 + 2 * pa[k]], dca = drow[5 + 2 * pa[k]];
                    const double dbb = drow[4 + 2 * pb[k]], dcb = drow[5 + 2 * pb[k]];
                    // d/dp of w (B_a^T D B_b), entry by entry
                    acc[k][0] += dwgt * (ba * d11 * bb + ca * d33 * cb) +
                                 wgt * (dba * d11 * bb + ba * d11 * dbb + dca * d33 * cb + ca * d33 * dcb);
                    acc[k][1] += dwgt * (ba * d12 * cb + ca * d33 * bb) +
                                 wgt * (dba * d12 * cb + ba * d12 * dcb + dca * d33 * bb + ca * d33 * dbb);
                    acc[k][2] += dwgt * (ca * d12 * bb + ba * d33 * cb) +
                                 wgt * (dca * d12 * bb + ca * d12 * dbb + dba * d33 * cb + ba * d33 * dcb);
                    acc[k][3] += dwgt * (ca * d11 * cb + ba * d33 * bb) +
                                 wgt * (dca * d11 * cb + ca * d11 * dcb + dba * d33 * bb + ba * d33 * dbb);
                }
            }
        }
        __syncwarp();
    }
    double part = 0.0;
#pragma unroll
    for (int k = 0; k < PPL; ++k) {
        if (lane + 32 * k < npairs) {
            const int ia = pa[k], ib = pb[k];
            const double ux = sU[w][2 * ib], uy = sU[w][2 * ib + 1];
            const double fx = acc[k][0] * ux + acc[k][1] * uy;
            const double fy = acc[k][2] * ux + acc[k][3] * uy;
            part += a.wsens[2 * sL[w][ia]] * fx + a.wsens[2 * sL[w][ia] + 1] * fy;
        }
    }
    // cohesive tractions at fixed U and committed state: the frame and the
    // length move, the opening follows the frame (dt = D d(delta))
    if (lane < 2 * T.n_coh) {
        const int ce = lane >> 1, q = lane & 1;
        const int c0 = T.coh_nodes[ce][0], c1 = T.coh_nodes[ce][1], c2 = T.coh_nodes[ce][2], c3 = T.coh_nodes[ce][3];
        const Dual x0{sX[w][c0], sDX[w][c0]}, x1{sX[w][c1], sDX[w][c1]};
        const Dual y0{sY[w][c0], sDY[w][c0]}, y1{sY[w][c1], sDY[w][c1]};
        const Dual jx = 0.5 * (x1 - x0), jy = 0.5 * (y1 - y0);
        const Dual mag = dsqrt(jx * jx + jy * jy);
        const Dual nx = -jy, ny = jx;
        const Dual dA = dsqrt(nx * nx + ny * ny);
        const Dual R00 = jx / mag, R01 = jy / mag, R10 = nx / dA, R11 = ny / dA;
        const double xi = q == 0 ? -0.57735026918962576450914878050196 : 0.57735026918962576450914878050196;
        const double N0 = 0.5 * (1.0 - xi), N1 = 0.5 * (1 + xi);
        double dg[2];
        for (int d = 0; d < 2; ++d)
            dg[d] = N0 * (sU[w][2 * c2 + d] - sU[w][2 * c0 + d]) + N1 * (sU[w][2 * c3 + d] - sU[w][2 * c1 + d]);
        const Dual dl0 = dg[0] * R00 + dg[1] * R01, dl1 = dg[0] * R10 + dg[1] * R11;
        double dl[2] = {dl0.v, dl1.v};
        const int qp = a.cut_coh_qp0[ci] + lane;
        double tr[2], Dc[2][2], dmax_t;
        cohesive_law(a.coh, a.dt, a.isv_c[qp], dl, tr, Dc, dmax_t);
        const double dtr0 = Dc[0][0] * dl0.d + Dc[0][1] * dl1.d;
        const double dtr1 = Dc[1][0] * dl0.d + Dc[1][1] * dl1.d;
        const Dual t0{tr[0], dtr0}, t1{tr[1], dtr1};
        const Dual tR0 = R00 * t0 + R10 * t1;
        const Dual tR1 = R01 * t0 + R11 * t1;
        if (dA.v != 0.0) {
            const Dual f0 = dA * tR0, f1 = dA * tR1;
            const int cn[4] = {c0, c1, c2, c3};
            const double Nn[2] = {N0, N1};
            for (int m = 0; m < 4; ++m) {
                const double sg = m < 2 ? -1.0 : 1.0;
                const int nd = sL[w][cn[m]];
                part += a.wsens[2 * nd] * (sg * Nn[m & 1] * f0.d) + a.wsens[2 * nd + 1] * (sg * Nn[m & 1] * f1.d);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(full, part, o);
    if (lane == 0) atomicAdd(&a.sens[param], part);
}

__global__ void k_to_fp32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n / 2; i += stride) {
        const double2 v = reinterpret_cast<const double2*>(a)[i];
        reinterpret_cast<float2*>(b)[i] = make_float2((float)v.x, (float)v.y);
    }
}




template <bool WANT_F, int TN>
void launch_tri_tn(const Ctx& c, const RowArgs& ra, cudaStream_t s) {
    const int n_tiles = (c.n_nodes + TN - 1) / TN;
    if (n_tiles <= 0) return;
    int grid = n_tiles;
    if (c.tuning.tri_persistent) {
        int per_sm = 0, dev = 0, n_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_assemble_tri<WANT_F, TN>, 2 * TN, 0);
        grid = std::min(n_tiles, std::max(1, per_sm) * n_sm);
    }
    k_assemble_tri<WANT_F, TN><<<grid, 2 * TN, 0, s>>>(ra, n_tiles);
}

void launch_tri(const Ctx& c, const RowArgs& ra, bool want_f, cudaStream_t s) {
    if (c.tuning.tri_grid && c.grid_emat) {
        launch_grid(c, ra.u, want_f, ra.want_K, s);
        return;
    }
    const int tn = kTriTileSizes[c.tuning.tri_variant];
    if (tn == 32) {
        if (want_f) launch_tri_tn<true, 32>(c, ra, s);
        else launch_tri_tn<false, 32>(c, ra, s);
    } else {
        if (want_f) launch_tri_tn<true, 64>(c, ra, s);
        else launch_tri_tn<false, 64>(c, ra, s);
    }
}

// Analytic shape-sensitivity passes (one launch per size class).
void launch_cut_sens_ad(const Ctx& c, const CutArgs& ca, cudaStream_t s) {
    for (int k = 0; k < kCutClasses; ++k) {
        const int n = c.cut_class_off[k + 1] - c.cut_class_off[k];
        if (n == 0) continue;
        CutArgs ck = ca;
        ck.n_cut = n;
        ck.first = c.cut_class_off[k];
        if (k == 0) k_cut_sens_ad<5, 1, 4><<<(n + 3) / 4, 128, 0, s>>>(ck);
        else if (k == 1) k_cut_sens_ad<7, 2, 4><<<(n + 3) / 4, 128, 0, s>>>(ck);
        else if (k == 2) k_cut_sens_ad<11, 4, 2><<<(n + 1) / 2, 64, 0, s>>>(ck);
        else k_cut_sens_ad<15, 8, 2><<<(n + 1) / 2, 64, 0, s>>>(ck);
    }
}

// Shape-sensitivity passes of the cut elements (one launch per size class).
void launch_cut_sens(const Ctx& c, const CutArgs& ca, cudaStream_t s) {
    for (int k = 0; k < kCutClasses; ++k) {
        const int n = c.cut_class_off[k + 1] - c.cut_class_off[k];
        if (n == 0) continue;
        CutArgs ck = ca;
        ck.n_cut = n;
        ck.first = c.cut_class_off[k];
        const int blocks = (n + 3) / 4;
        if (k == 0) k_cut_sens<5, 1, 4><<<blocks, 128, 0, s>>>(ck);
        else if (k == 1) k_cut_sens<7, 2, 4><<<blocks, 128, 0, s>>>(ck);
        else if (k == 2) k_cut_sens<11, 4, 4><<<blocks, 128, 0, s>>>(ck);
        else k_cut_sens<15, 8, 4><<<blocks, 128, 0, s>>>(ck);
    }
}

RowArgs row_args(const Ctx& c, const double* U, bool want_f, bool want_K) {
    RowArgs ra;
    ra.n_nodes = c.n_nodes;
    ra.n_reg = c.n_reg;
    ra.row_ptr = c.row_ptr;
    ra.col = c.col;
    ra.ne_ptr = c.ne_ptr;
    ra.ne_list = c.ne_list;
    ra.tri_map = c.tri_map[c.tuning.tri_variant];
    ra.diag = c.diag;
    ra.elem4 = c.elem4;
    ra.x = c.x;
    ra.y = c.y;
    ra.u = U;
    ra.dmat = c.dmat;
    ra.n_mat = (int)c.hm.spec.materials.size();
    ra.K = c.K;
    ra.f = c.F;
    ra.want_K = want_K;
    ra.want_f = want_f;
    return ra;
}

CutArgs cut_args(const Ctx& c, const double* U, double dt) {
    CutArgs ca{};
    ca.n_cut = c.n_cut;
    ca.first = 0;
    ca.cut_nodes = c.cut_nodes;
    ca.cut_tmpl = c.cut_tmpl;
    ca.cut_child_mat = c.cut_child_mat;
    ca.cut_coh_qp0 = c.cut_coh_qp0;
    ca.x = c.x;
    ca.y = c.y;
    ca.u = U;
    ca.dmat = c.dmat;
    ca.isv_c = c.isv_c;
    ca.coh = c.coh;
    ca.dt = dt;
    return ca;
}

// Launches kern with the programmatic-stream-serialization attribute (see
// pdl_trigger / pdl_wait).
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), int grid, int block, size_t smem, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
}

void launch_cut_points(const Ctx& c, cudaStream_t s) {
    if (c.n_cut_pts > 0)
        launch_pdl(k_cut_points, (c.n_cut_pts + kPointThreads - 1) / kPointThreads, kPointThreads, 0, s, c.n_cut_pts,
                   reinterpret_cast<const int4*>(c.cut_pts), c.x, c.y, c.dmat, c.cut_rows);
}

void launch_coh_points(const Ctx& c, const double* U, double dt, cudaStream_t s) {
    if (c.n_coh_qp <= 0) return;
    CohArgs ca;
    ca.n_qp = c.n_coh_qp;
    ca.coh_rec = c.coh_rec;
    ca.cut_nodes = c.cut_nodes;
    ca.cut_tmpl = c.cut_tmpl;
    ca.x = c.x;
    ca.y = c.y;
    ca.u = U;
    ca.isv_c = c.isv_c;
    ca.isv_t = c.isv_t;
    ca.coh_rows = c.coh_rows;
    ca.coh = c.coh;
    ca.dt = dt;
    launch_pdl(k_coh_points, (c.n_coh_qp + 127) / 128, 128, 0, s, ca);
}

template <int NL, bool WF, bool COH>
int launch_elems_inst(const ElemArgs& ea, int blocks, int bs, size_t smem, cudaStream_t s) {
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k_cut_elems<NL, WF, COH>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_fail(e, "k_cut_elems shared memory");
    }
    launch_pdl(k_cut_elems<NL, WF, COH>, blocks, bs, smem, s, ea);
    return PG_OK;
}

// residual passes (WF) and cohesive meshes (COH) take their own instances, so
// that the stiffness-only pass of a linear mesh carries neither in registers
template <int NL>
int launch_elems_nl(const ElemArgs& ea, bool coh, int blocks, int bs, size_t smem, cudaStream_t s) {
    if (ea.want_f) {
        return coh ? launch_elems_inst<NL, true, true>(ea, blocks, bs, smem, s)
                   : launch_elems_inst<NL, true, false>(ea, blocks, bs, smem, s);
    }
    return coh ? launch_elems_inst<NL, false, true>(ea, blocks, bs, smem, s)
               : launch_elems_inst<NL, false, false>(ea, blocks, bs, smem, s);
}

// one launch per size class; cut_warps x 32 threads per CTA.  direct: the
// blocks of one-contribution slots go into K (the triangle kernel runs
// before on the same stream); otherwise every block goes to fold order.
int launch_cut_elems(const Ctx& c, const double* U, bool want_f, bool want_K, bool direct, cudaStream_t s) {
    ElemArgs ea;
    ea.cut_nodes = c.cut_nodes;
    ea.cut_tmpl = c.cut_tmpl;
    ea.cut_coh_qp0 = c.cut_coh_qp0;
    ea.cut_slot_ptr = c.cut_slot_ptr;
    ea.kpos = c.cut_kpos;
    ea.kdir = c.cut_kdir;
    ea.fpos = c.cut_fpos;
    ea.pts = reinterpret_cast<const int4*>(c.cut_pts);
    ea.pt_off = c.cut_pt_off;
    ea.row_off = c.cut_row_off;
    ea.x = c.x;
    ea.y = c.y;
    ea.dmat = c.dmat;
    ea.coh_rows = c.coh_rows;
    ea.u = U;
    ea.ke = c.cut_ke;
    ea.fe = c.cut_fe;
    ea.K = c.K;
    ea.want_K = want_K;
    ea.want_f = want_f;
    ea.direct = direct ? 1 : 0;
    const int w = c.tuning.cut_warps == 2 ? 0 : c.tuning.cut_warps == 8 ? 2 : 1;
    const int bs = 32 * kCutCtaWarps[w];
    for (int k = 0; k < kCutClasses; ++k) {
        const int n = c.cut_class_off[k + 1] - c.cut_class_off[k];
        if (n == 0) continue;
        ea.n_elem = n;
        ea.first = c.cut_class_off[k];
        const int epc = cut_elems_per_cta(bs, kCutClassNl[k]);
        const int blocks = (n + epc - 1) / epc;
        const size_t smem = sizeof(double) * (size_t)std::max(2, c.cut_span[k][w]);
        if (smem > 227 * 1024) {
            set_error("cut elements: a CTA's quadrature rows exceed the shared memory (use fewer warps per CTA)");
            return PG_ERR_LIMIT;
        }
        int rc;
        const bool coh = c.n_coh_qp > 0;
        if (k == 0) rc = launch_elems_nl<5>(ea, coh, blocks, bs, smem, s);
        else if (k == 1) rc = launch_elems_nl<7>(ea, coh, blocks, bs, smem, s);
        else if (k == 2) rc = launch_elems_nl<11>(ea, coh, blocks, bs, smem, s);
        else rc = launch_elems_nl<15>(ea, coh, blocks, bs, smem, s);
        if (rc != PG_OK) return rc;
    }
    return PG_OK;
}

// direct: fold only the runs of two or more blocks (launch_cut_elems stored the others)
void launch_cut_fold(const Ctx& c, bool want_f, bool want_K, bool direct, cudaStream_t s) {
    const int nK = direct ? c.n_fold_Km : c.n_fold_K;
    if (want_K && nK > 0)
        launch_pdl(k_fold_K, (nK + 255) / 256, 256, 0, s, nK, direct ? c.fold_Km_slot : c.fold_K_slot, c.fold_K_ptr,
                   direct ? c.fold_Km_rng : nullptr, c.cut_ke, c.K);
    if (want_f && c.n_fold_f > 0)
        launch_pdl(k_fold_f, (c.n_fold_f + 255) / 256, 256, 0, s, c.n_fold_f, c.fold_f_node, c.fold_f_ptr, c.cut_fe,
                   c.F);
}

// the cut elements' whole pass after the triangle kernel on stream s
int launch_cut_all(const Ctx& c, const double* U, double dt, bool want_f, bool want_K, cudaStream_t s) {
    launch_coh_points(c, U, dt, s);
    const int rc = launch_cut_elems(c, U, want_f, want_K, true, s);
    if (rc != PG_OK) return rc;
    launch_cut_fold(c, want_f, want_K, true, s);
    return PG_OK;
}

int launch_assemble(Ctx& c, const double* U, double dt, bool want_f, bool want_K, cudaStream_t s) {
    // The triangle kernel writes every regular-element value of K (and f)
    // once; then the cut elements' cohesive points, quadrature rows and
    // blocks are formed, the blocks of slots no other contribution reaches
    // go into K, and the fold adds the rest to the rows they touch and writes
    // the remaining enrichment rows and columns whole.  Nothing needs
    // clearing first.  One stream, the kernels chained by programmatic
    // dependent launch, unless the tuning sets cut_overlap with the grid
    // kernel (the persistent one then leaves that many CTA slots per SM):
    // then the cut elements' kernels run on the second stream beside it,
    // every block goes to fold order, and the fold waits for both.
    if (!(c.tuning.tri_grid && c.grid_emat)) {
        const int rc = ensure_tri_map(c);
        if (rc != PG_OK) return rc;
    }
    const RowArgs ra = row_args(c, U, want_f, want_K);
    if (c.timing) cudaEventRecord(c.ea0, s);
    const bool overlap = c.n_cut > 0 && c.tuning.cut_overlap > 0 && c.tuning.tri_grid && c.grid_emat &&
                         !(c.timing && c.timing_split);
    if (overlap) {
        // the cut elements' rows and pairs on the second stream, beside the
        // persistent grid kernel (which leaves them CTA slots); the fold joins
        PG_CUDA(cudaEventRecord(c.fork_ev, s));
        PG_CUDA(cudaStreamWaitEvent(c.aux, c.fork_ev, 0));
        launch_coh_points(c, U, dt, c.aux);
        const int rc = launch_cut_elems(c, U, want_f, want_K, false, c.aux);
        if (rc != PG_OK) return rc;
        PG_CUDA(cudaEventRecord(c.join_ev, c.aux));
        launch_tri(c, ra, want_f, s);
        PG_CUDA(cudaStreamWaitEvent(s, c.join_ev, 0));
        launch_cut_fold(c, want_f, want_K, false, s);
        PG_CUDA(cudaGetLastError());
        if (c.timing) cudaEventRecord(c.ea2, s);
        return PG_OK;
    }
    launch_tri(c, ra, want_f, s);
    PG_CUDA(cudaGetLastError());
    if (c.timing && c.timing_split) cudaEventRecord(c.ea1, s);
    if (c.n_cut > 0) {
        const int rc = launch_cut_all(c, U, dt, want_f, want_K, s);
        if (rc != PG_OK) return rc;
        PG_CUDA(cudaGetLastError());
    }
    if (c.timing) cudaEventRecord(c.ea2, s);
    return PG_OK;
}

// Times every launch shape of the two assembly stages on this mesh (L2
// flushed before each launch, `reps` launches each, device events) and
// keeps the fastest of each in c.tuning.  ms_tri: the row-tile kernel with
// 32 / 64 node rows per CTA, one CTA per tile / persistent (4 values), then
// the structured-grid kernel (the fastest of 128 and 256 threads per CTA,
// one CTA per tile or persistent and pipelined; 0 without a structured grid); ms_cut: the cut elements' work on one stream
// (cohesive points, rows and blocks, the fold) with 2 / 4 / 8 warps per
// k_cut_elems CTA.
// K is left undefined: the next solve reassembles.
int autotune_assembly(Ctx& c, int reps, float* ms_tri, float* ms_cut) {
    cudaStream_t s = c.stream;
    reps = std::max(1, reps);
    const size_t flush_bytes = 256u << 20;  // twice the L2
    void* flush = nullptr;
    PG_CUDA(cudaMalloc(&flush, flush_bytes));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto timed = [&](auto&& launch) -> float {
        launch();  // warm-up (first-launch costs)
        float total = 0.f;
        for (int r = 0; r < reps; ++r) {
            cudaMemsetAsync(flush, r & 0xff, flush_bytes, s);
            cudaEventRecord(e0, s);
            launch();
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            total += ms;
        }
        return total / reps;
    };
    AsmTuning best = c.tuning;
    float best_tri = 1e30f, best_cut = 1e30f;
    int idx = 0;
    const int trc = ensure_tri_map(c);
    if (trc != PG_OK) return trc;
    c.tuning.tri_grid = 0;
    for (int v = 0; v < kTriTileVariants; ++v)
        for (int p = 0; p < 2; ++p, ++idx) {
            c.tuning.tri_variant = v;
            c.tuning.tri_persistent = p;
            const RowArgs ra = row_args(c, c.U, false, true);
            const float ms = timed([&] { launch_tri(c, ra, false, s); });
            if (ms_tri) ms_tri[idx] = ms;
            if (ms < best_tri) {
                best_tri = ms;
                best.tri_variant = v;
                best.tri_persistent = p;
                best.tri_grid = 0;
            }
        }
    // the fastest CTA size of the grid kernel per variant (one CTA per tile, persistent)
    float grid_ms_of[2] = {1e30f, 1e30f};
    int grid_bs_of[2] = {256, 256};
    if (c.grid_emat) {
        c.tuning.tri_grid = 1;
        float ms_grid = 0.f;
        for (int bs : {128, 256})
            for (int p = 0; p < 2; ++p) {
                c.tuning.grid_block = bs;
                c.tuning.tri_persistent = p;  // 1: the persistent, pipelined grid kernel
                const RowArgs ra = row_args(c, c.U, false, true);
                const float ms = timed([&] { launch_tri(c, ra, false, s); });
                if (ms < grid_ms_of[p]) {
                    grid_ms_of[p] = ms;
                    grid_bs_of[p] = bs;
                }
                if (ms_grid == 0.f || ms < ms_grid) ms_grid = ms;
                if (ms < best_tri) {
                    best_tri = ms;
                    best.tri_grid = 1;
                    best.grid_block = bs;
                    best.tri_persistent = p;
                }
            }
        if (ms_tri) ms_tri[4] = ms_grid;
    } else if (ms_tri) {
        ms_tri[4] = 0.f;
    }
    const int warps[3] = {2, 4, 8};
    for (int k = 0; k < 3; ++k) {
        c.tuning.cut_warps = warps[k];
        float ms = 0.f;
        int rc = PG_OK;
        if (c.n_cut > 0) ms = timed([&] { rc = launch_cut_all(c, c.U, 1.0, false, true, s); });
        if (rc != PG_OK) {
            cudaFree(flush);
            return rc;
        }
        if (ms_cut) ms_cut[k] = ms;
        if (ms < best_cut) {
            best_cut = ms;
            best.cut_warps = warps[k];
        }
    }
    // with the grid kernel, whole passes decide: each variant of it (its
    // fastest CTA size) with the cut elements' kernels after it on the same
    // stream, or beside it on the second stream -- the persistent one leaving
    // them 1 or 2 CTA slots per SM
    best.cut_overlap = 0;
    if (c.n_cut > 0 && best.tri_grid && c.grid_emat) {
        float best_pass = 1e30f;
        AsmTuning pick = best;
        for (int p = 0; p < 2; ++p)
            for (int ov = 0; ov <= (p ? 2 : 1); ++ov) {
                c.tuning = best;
                c.tuning.tri_persistent = p;
                c.tuning.grid_block = grid_bs_of[p];
                c.tuning.cut_overlap = ov;
                const float ms = timed([&] { launch_assemble(c, c.U, 1.0, false, true, s); });
                if (ms < best_pass) {
                    best_pass = ms;
                    pick = c.tuning;
                }
            }
        best = pick;
    }
    c.tuning = best;
    c.assembled = false;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(flush);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

// ---------------------------------------------------------------------------
// Stress and strain recovery (Problem::compute_stress_strain,
// src/Problem.cpp:428-534) and the homogenised response
// ---------------------------------------------------------------------------
// At every volumetric quadrature point, element by element in the
// reference's point order: strain = B u (Voigt, engineering shear), stress
// = D strain, and the point's J W.  Uncut elements have the four points of
// the Tri3 rule (their strain is constant); a cut element has its children's
// points in template order -- a Tri3 child's four points share one strain,
// which the device forms once from the child's quadrature row.  A point of
// zero weight (a collapsed child) has no defined gradients: its strain and
// stress are NaN, as the reference's inverse map leaves them.
__constant__ double kTri3W[4] = {-0.28125, 0.260416666666666666666666666666665, 0.260416666666666666666666666666665,
                              0.260416666666666666666666666666665};  // tri3.cpp:107-115

__device__ __forceinline__ void voigt_stress(const double e[3], double d11, double d12, double d33, double s[3]) {
    s[0] = d11 * e[0] + d12 * e[1];
    s[1] = d12 * e[0] + d11 * e[1];
    s[2] = d33 * e[2];
}

// out: 7 FP64 per point {strain 3, stress 3, J W}
__global__ void k_stress_uncut(int n_elem, const int4* __restrict__ elem4, const int* __restrict__ elem_cut,
                               const int* __restrict__ qp_off, const double* __restrict__ x,
                               const double* __restrict__ y, const double* __restrict__ u,
                               const double* __restrict__ dmat, double* out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elem || elem_cut[e] >= 0) return;
    const int4 el = __ldg(&elem4[e]);
    const int n[3] = {el.x, el.y, el.z};
    double X[3], Y[3], ux[3], uy[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        X[v] = __ldg(&x[n[v]]);
        Y[v] = __ldg(&y[n[v]]);
        ux[v] = __ldg(&u[2 * n[v]]);
        uy[v] = __ldg(&u[2 * n[v] + 1]);
    }
    const double J = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0]);
    const double iJ = 1.0 / J;
    const double b[3] = {(Y[1] - Y[2]) * iJ, (Y[2] - Y[0]) * iJ, (Y[0] - Y[1]) * iJ};
    const double c[3] = {(X[2] - X[1]) * iJ, (X[0] - X[2]) * iJ, (X[1] - X[0]) * iJ};
    double eps[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        eps[0] += b[v] * ux[v];
        eps[1] += c[v] * uy[v];
        eps[2] += c[v] * ux[v] + b[v] * uy[v];
    }
    double sig[3];
    voigt_stress(eps, __ldg(&dmat[3 * el.w]), __ldg(&dmat[3 * el.w + 1]), __ldg(&dmat[3 * el.w + 2]), sig);
    double* o = out + 7 * (size_t)__ldg(&qp_off[e]);
    for (int q = 0; q < 4; ++q, o += 7) {
        o[0] = eps[0]; o[1] = eps[1]; o[2] = eps[2];
        o[3] = sig[0]; o[4] = sig[1]; o[5] = sig[2];
        o[6] = J * kTri3W[q];
    }
}

static_assert(kCutClasses == 4, "c_class_nl lists the classes one by one");
__constant__ int c_class_nl[kCutClasses] = {kCutClassNl[0], kCutClassNl[1], kCutClassNl[2], kCutClassNl[3]};

// one thread per cut element (class order), from its quadrature rows
// (k_cut_points, point-major); elem_of: class order -> mesh element
__global__ void k_stress_cut(int n_cut, const int* __restrict__ class_off, const int* __restrict__ elem_of,
                             const int* __restrict__ cut_tmpl, const int* __restrict__ cut_nodes,
                             const long long* __restrict__ row_off, const double* __restrict__ rows,
                             const double* __restrict__ u, const int* __restrict__ qp_off, double* out) {
    const int oi = blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= n_cut) return;
    int k = 0;
    while (k < kCutClasses - 1 && oi >= class_off[k + 1]) ++k;
    const int W = 4 + 2 * c_class_nl[k];
    const DevTemplate& T = c_tmpl[cut_tmpl[oi]];
    const int nl = 3 + T.n_enr;
    const double* rw = rows + row_off[oi];
    double* o = out + 7 * (size_t)qp_off[elem_of[oi]];
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int ch = 0; ch < T.n_child; ++ch) {
        const int type = T.child_type[ch];
        const int nq_dev = c_quad[type].nq;          // points the device forms
        const int nq_ref = type == kChildTri3 ? 4 : nq_dev;
        for (int q = 0; q < nq_dev; ++q, rw += W) {
            const double wgt = rw[0];
            double eps[3] = {0.0, 0.0, 0.0}, sig[3];
            if (wgt != 0.0) {
                for (int l = 0; l < nl; ++l) {
                    const int nd = cut_nodes[(size_t)kCutNodeStride * oi + l];
                    const double gx = rw[4 + 2 * l], gy = rw[5 + 2 * l];
                    const double ux = u[2 * nd], uy = u[2 * nd + 1];
                    eps[0] += gx * ux;
                    eps[1] += gy * uy;
                    eps[2] += gy * ux + gx * uy;
                }
                voigt_stress(eps, rw[1], rw[2], rw[3], sig);
            } else {
                eps[0] = eps[1] = eps[2] = sig[0] = sig[1] = sig[2] = nan;
            }
            // a Tri3 child's single device point stands for the rule's four
            const int reps = type == kChildTri3 ? nq_ref : 1;
            for (int r = 0; r < reps; ++r, o += 7) {
                o[0] = eps[0]; o[1] = eps[1]; o[2] = eps[2];
                o[3] = sig[0]; o[4] = sig[1]; o[5] = sig[2];
                // J W of the point: the Tri3 child's row carries det x the rule's summed weight
                o[6] = type == kChildTri3 ? wgt / c_quad[kChildTri3].w[0] * kTri3W[r] : wgt;
            }
        }
    }
}

// per CTA: sums over its points of J W (strain, stress) and J W, skipping
// points of zero weight; the CTAs' partials are added in order afterwards
__global__ void __launch_bounds__(256) k_stress_partial(long long n_pts, const double* __restrict__ out,
                                                        double* partial) {
    __shared__ double sm[7][256];
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    for (long long p = blockIdx.x * 256LL + threadIdx.x; p < n_pts; p += 256LL * gridDim.x) {
        const double* o = out + 7 * p;
        const double w = o[6];
        if (w == 0.0) continue;
        for (int k = 0; k < 6; ++k) acc[k] += w * o[k];
        acc[6] += w;
    }
    for (int k = 0; k < 7; ++k) sm[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int k = 0; k < 7; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x < 7) partial[7 * (size_t)blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

// Point offsets and the tables the recovery needs, built on its first call.
int stress_prepare(Ctx& c) {
    if (c.qp_off) return PG_OK;
    const HostMesh& hm = c.hm;
    std::vector<int> off(hm.n_elem + 1, 0);
    for (int e = 0; e < hm.n_elem; ++e) {
        int n = 4;
        const int ci = hm.elem_cut[e];
        if (ci >= 0) {
            const CutTemplate& T = cut_template(hm.cut_tmpl[ci]);
            n = 0;
            for (int ch = 0; ch < T.n_child; ++ch) {
                const int nc = T.child_n[ch];
                n += child_quadrature(nc == 3 ? kChildTri3 : nc == 4 ? kChildQuad4 : nc == 5 ? kChildPoly5 : kChildPoly6).nq;
            }
        }
        off[e + 1] = off[e] + n;
    }
    // class order -> mesh element (the order ctx_create gives the cut arrays)
    std::vector<int> elem_of;
    for (int k = 0; k < kCutClasses; ++k) {
        const int lo = k == 0 ? 0 : kCutClassNl[k - 1];
        for (int ci = 0; ci < hm.n_cut; ++ci) {
            const int nl = 3 + cut_template(hm.cut_tmpl[ci]).n_enr;
            if (nl > lo && nl <= kCutClassNl[k]) elem_of.push_back(hm.cut_elem[ci]);
        }
    }
    c.n_qp_total = off.back();
    auto up = [&](auto** dst, const auto& v) -> int {
        using T = std::remove_pointer_t<std::remove_reference_t<decltype(*dst)>>;
        PG_CUDA(cudaMalloc((void**)dst, std::max<size_t>(1, v.size()) * sizeof(T)));
        if (!v.empty()) PG_CUDA(h2d_sync(*dst, v.data(), v.size() * sizeof(T)));
        return PG_OK;
    };
    int rc;
    if ((rc = up(&c.qp_off, off)) || (rc = up(&c.qp_elem_cut, hm.elem_cut)) || (rc = up(&c.qp_cut_elem, elem_of)) ||
        (rc = up(&c.qp_class_off, std::vector<int>(c.cut_class_off, c.cut_class_off + kCutClasses + 1))))
        return rc;
    PG_CUDA(cudaMalloc((void**)&c.qp_out, 7 * std::max<size_t>(1, (size_t)c.n_qp_total) * sizeof(double)));
    if (c.n_cut > 0 && !c.cut_rows)
        PG_CUDA(cudaMalloc((void**)&c.cut_rows, std::max<size_t>(1, (size_t)c.cut_rows_len) * sizeof(double)));
    return PG_OK;
}

// Runs the recovery on stream s; mean7 (host, nullable): J W-weighted sums of
// strain (3) and stress (3) divided by the total J W, then that total.
int stress_strain(Ctx& c, const double* U, cudaStream_t s, double* mean7) {
    int rc = stress_prepare(c);
    if (rc != PG_OK) return rc;
    k_stress_uncut<<<(c.n_elem + 255) / 256, 256, 0, s>>>(c.n_elem, c.elem4, c.qp_elem_cut, c.qp_off, c.x, c.y, U,
                                                          c.dmat, c.qp_out);
    if (c.n_cut > 0) {
        launch_cut_points(c, s);
        k_stress_cut<<<(c.n_cut + 127) / 128, 128, 0, s>>>(c.n_cut, c.qp_class_off, c.qp_cut_elem, c.cut_tmpl,
                                                           c.cut_nodes, c.cut_row_off, c.cut_rows, U, c.qp_off,
                                                           c.qp_out);
    }
    PG_CUDA(cudaGetLastError());
    if (mean7) {
        constexpr int kParts = 148 * 4;
        double* part = nullptr;
        PG_CUDA(cudaMallocAsync((void**)&part, 7 * kParts * sizeof(double), s));
        k_stress_partial<<<kParts, 256, 0, s>>>(c.n_qp_total, c.qp_out, part);
        std::vector<double> hp(7 * kParts);
        PG_CUDA(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        PG_CUDA(cudaStreamSynchronize(s));
        cudaFreeAsync(part, s);
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int b = 0; b < kParts; ++b)
            for (int k = 0; k < 7; ++k) acc[k] += hp[7 * b + k];
        for (int k = 0; k < 6; ++k) mean7[k] = acc[6] != 0.0 ? acc[k] / acc[6] : 0.0;
        mean7[6] = acc[6];
    }
    return PG_OK;
}

int launch_to_fp32(Ctx& c, cudaStream_t s) {
    const size_t n = 4 * (size_t)c.n_blocks;
    k_to_fp32<<<148 * 8, 256, 0, s>>>(c.K, c.Kf, n);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pgb
