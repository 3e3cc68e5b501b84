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

// Quadrature rows of every cut element, one thread per point.  What a point
// needs of the mesh is static, so the host packs it into one 64-byte record
// (kCutPointInts ints, see build_cut_points): the thread reads its record,
// then the coordinates it names, and writes its row.  It runs on a second
// stream beside the structured-grid kernel.
struct CutPointArgs {
    int n_pts;
    const int4* __restrict__ pts;
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ dmat;
    double* rows;
};

__global__ void __launch_bounds__(256) k_cut_points(CutPointArgs a) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.n_pts) return;
    const int4* rec = a.pts + 4 * (size_t)p;
    const int4 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3);
    const int gn[kMaxChildNodes] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y};
    const int mat = r2.y, lnp = r2.z, meta = r2.w;
    const int q = meta & 255, type = (meta >> 8) & 3, nc = (meta >> 10) & 7, nl = (meta >> 13) & 15;
    const long long base = (long long)(unsigned)r3.x | ((long long)r3.y << 32);
    const int nq_e = r3.z, l = r3.w;
    int ln[kMaxChildNodes];
    double cx[kMaxChildNodes], cy[kMaxChildNodes];
#pragma unroll
    for (int k = 0; k < kMaxChildNodes; ++k) {
        ln[k] = (lnp >> (4 * k)) & 15;
        cx[k] = cy[k] = 0.0;
        if (k < nc) {
            cx[k] = __ldg(&a.x[gn[k]]);
            cy[k] = __ldg(&a.y[gn[k]]);
        }
    }
    const double PX[3] = {__ldg(&a.x[r1.z]), __ldg(&a.x[r1.w]), __ldg(&a.x[r2.x])};
    const double PY[3] = {__ldg(&a.y[r1.z]), __ldg(&a.y[r1.w]), __ldg(&a.y[r2.x])};
    double pbx[3], pby[3];
    parent_gradients(PX, PY, pbx, pby);
    const double dm[3] = {__ldg(&a.dmat[3 * mat]), __ldg(&a.dmat[3 * mat + 1]), __ldg(&a.dmat[3 * mat + 2])};
    cut_row(a.rows + base + l, nq_e, nl, g_quad[type], q, nc, ln, cx, cy, dm, pbx, pby);
}

// Point records of k_cut_points, per point kCutPointInts ints: global nodes of
// its child (6, unused ones repeat the first), of the parent (3), the child's
// material, the child nodes' local numbers (4 bits each), then point q (8
// bits), child type (2), child node count (3) and the element's local-function
// count (4), then the element's first row offset in doubles (2 ints, low
// first), its point count and this point's number within it.  An element's
// rows are stored value-major (value j of point l at j nq + l), so that the
// threads of consecutive points write consecutive doubles.  Points are in
// class order, each element's in the order of its rows.
void build_cut_points(const std::vector<int>& nodes, const std::vector<int>& tmpl, const std::vector<int>& chm,
                      const std::vector<long long>& roff, const int* class_off, std::vector<int>& out) {
    out.clear();
    for (int k = 0; k < kCutClasses; ++k)
        for (int oi = class_off[k]; oi < class_off[k + 1]; ++oi) {
            const CutTemplate& T = cut_template(tmpl[oi]);
            const int* en = &nodes[(size_t)kCutNodeStride * oi];
            const int nq_e = device_point_count(tmpl[oi]);
            int l = 0;
            for (int ch = 0; ch < T.n_child; ++ch) {
                const int nc = T.child_n[ch];
                const int type = nc == 3 ? kChildTri3 : nc == 4 ? kChildQuad4 : nc == 5 ? kChildPoly5 : kChildPoly6;
                int lnp = 0;
                for (int c = 0; c < nc; ++c) lnp |= T.child_nodes[ch][c] << (4 * c);
                for (int q = 0; q < device_child_nq(type); ++q, ++l) {
                    int r[kCutPointInts] = {};
                    for (int c = 0; c < kMaxChildNodes; ++c) r[c] = en[c < nc ? T.child_nodes[ch][c] : 0];
                    r[6] = en[0];
                    r[7] = en[1];
                    r[8] = en[2];
                    r[9] = chm[(size_t)kMaxChildren * oi + ch];
                    r[10] = lnp;
                    r[11] = q | (type << 8) | (nc << 10) | ((3 + T.n_enr) << 13);
                    r[12] = (int)(unsigned)(roff[oi] & 0xffffffffLL);
                    r[13] = (int)(roff[oi] >> 32);
                    r[14] = nq_e;
                    r[15] = l;
                    out.insert(out.end(), r, r + kCutPointInts);
                }
            }
        }
}

// Per-warp shared tables: one row per quadrature point of the current chunk
// holding {wgt, d11, d12, d33, (gx, gy) of every local function}, and one
// row per cohesive point holding {wgt, N0, N1, (R^T D R) 4, (R^T t) 2}.
// NL is the size class's largest local node count; PPL = ceil(NL^2 / 32)
// node-pair blocks per lane.
constexpr int kQpChunk = 32;
constexpr int kCRow = 10;

template <int NL, int PPL, int W, bool SENS = false>
__global__ void __launch_bounds__(32 * W, (NL <= 5 ? (SENS ? 24 : 32) : (NL <= 7 ? 16 : 8)) / W) k_assemble_cut(CutArgs a) {
    constexpr int kCutWarps = W;
    constexpr int kQRow = 4 + 2 * NL;
    __shared__ double sX[kCutWarps][NL], sY[kCutWarps][NL];
    __shared__ double sU[kCutWarps][2 * NL];
    __shared__ int sL[kCutWarps][NL];
    __shared__ double sQ[kCutWarps][kQpChunk][kQRow];
    __shared__ double sC[kCutWarps][2 * kMaxCoh][kCRow];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int oi = blockIdx.x * kCutWarps + w;
    if (oi >= a.n_cut) return;
    const int ci = a.first + oi;  // class-ordered element index
    // the node list (padded with -1), the template and the slot pointer do
    // not depend on each other: their loads go out together
    const int node = lane < NL ? __ldg(&a.cut_nodes[kCutNodeStride * ci + lane]) : -1;
    const int tmpl = __ldg(&a.cut_tmpl[ci]);
    const int slot0 = __ldg(&a.cut_slot_ptr[ci]);
    const long long roff = SENS ? 0 : __ldg(&a.row_off[ci]);
    const DevTemplate& T = c_tmpl[tmpl];
    const int nl = 3 + T.n_enr;
    // the element's block slots are needed only at the end: issue their loads now
    const int* slots = a.cut_slot + slot0;
    int slot[PPL];
#pragma unroll
    for (int k = 0; k < PPL; ++k)
        slot[k] = (!SENS && a.want_K && lane + 32 * k < nl * nl) ? __ldg(&slots[lane + 32 * k]) : -1;
    if (lane < nl) {
        sL[w][lane] = node;
        if (SENS || T.n_coh > 0) {  // otherwise the quadrature rows carry all the geometry
            sX[w][lane] = a.x[node];
            sY[w][lane] = a.y[node];
        }
        if (SENS || a.want_f || T.n_coh > 0) {
            sU[w][2 * lane] = a.u[2 * node];
            sU[w][2 * lane + 1] = a.u[2 * node + 1];
        }
    }
    __syncwarp();
    double part = 0.0;    // SENS: this lane's share of wsens . f_e
    int sel = -1;         // SENS: the inclusion whose radius moves
    double hstep = 0.0;
    if (SENS) {
        const unsigned full = 0xffffffffu;
        const int my_inc = (lane >= 3 && lane < nl) ? a.node_inc[sL[w][lane]] : -1;
        // the which-th distinct inclusion among the enrichment slots, in slot order
        int count = 0;
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
        hstep = a.h_rel * a.radius[sel];
        if (lane < nl && my_inc == sel) {
            const int node = sL[w][lane];
            sX[w][lane] += a.sgn * hstep * a.vel[2 * node];
            sY[w][lane] += a.sgn * hstep * a.vel[2 * node + 1];
        }
        __syncwarp();
    }
    // parent (Tri3) gradients are constant over the element (SENS: its nodes have moved)
    double pbx[3] = {0.0, 0.0, 0.0}, pby[3] = {0.0, 0.0, 0.0};
    if (SENS) parent_gradients(sX[w], sY[w], pbx, pby);

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
        if (SENS) {
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
        } else {
            // the chunk's rows, formed by k_cut_points (value-major: value j of
            // point q at j nq_total + q): a coalesced read, transposed into sQ
            const int nqc = min(kQpChunk, nq_total - qbase);
            const double* src = a.rows + roff + qbase;
            for (int i = lane; i < nqc * kQRow; i += 32) {
                const int j = i / nqc, q = i - j * nqc;
                sQ[w][q][j] = __ldg(&src[(long long)j * nq_total + q]);
            }
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
    // bulk internal force f_a = sum_b K_ab u_b
    if (SENS || a.want_f) {
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
            if (lane + 32 * k < npairs) {
                const int ia = pa[k], ib = pb[k];
                const double ux = sU[w][2 * ib], uy = sU[w][2 * ib + 1];
                const double fx = acc[k][0] * ux + acc[k][1] * uy;
                const double fy = acc[k][2] * ux + acc[k][3] * uy;
                if (SENS) {
                    part += a.wsens[2 * sL[w][ia]] * fx + a.wsens[2 * sL[w][ia] + 1] * fy;
                } else {
                    atomicAdd(&a.f[2 * sL[w][ia]], fx);
                    atomicAdd(&a.f[2 * sL[w][ia] + 1], fy);
                }
            }
        }
    }
    if (T.n_coh == 0) goto scatter;
    // cohesive sub-elements: two Gauss points each (CohEdge2, w = 1), one lane per point
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
        const double dmax_c = a.isv_c[qp];
        double tr[2], Dc[2][2], dmax_t;
        cohesive_law(a.coh, a.dt, dmax_c, dl, tr, Dc, dmax_t);
        if (!SENS) a.isv_t[qp] = dmax_t;
        double* row = sC[w][lane];
        row[0] = dA * 1.0;
        row[1] = N0;
        row[2] = N1;
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                double s = 0.0;
                for (int k1 = 0; k1 < 2; ++k1)
                    for (int k2 = 0; k2 < 2; ++k2) s += R[k1][i] * Dc[k1][k2] * R[k2][j];
                row[3 + 2 * i + j] = s;
            }
        const double tR0 = R[0][0] * tr[0] + R[1][0] * tr[1];
        const double tR1 = R[0][1] * tr[0] + R[1][1] * tr[1];
        row[7] = tR0;
        row[8] = tR1;
        const double wgt = row[0];
        if ((SENS || a.want_f) && wgt != 0.0) {
            const int cn[4] = {c0, c1, c2, c3};
            const double Nn[2] = {N0, N1};
            for (int m = 0; m < 4; ++m) {
                const double sgn = m < 2 ? -1.0 : 1.0;
                const int node = sL[w][cn[m]];
                if (SENS) {
                    part += a.wsens[2 * node] * (wgt * sgn * Nn[m & 1] * tR0) +
                            a.wsens[2 * node + 1] * (wgt * sgn * Nn[m & 1] * tR1);
                } else {
                    atomicAdd(&a.f[2 * node], wgt * sgn * Nn[m & 1] * tR0);
                    atomicAdd(&a.f[2 * node + 1], wgt * sgn * Nn[m & 1] * tR1);
                }
            }
        }
    }
    __syncwarp();
    if (a.want_K) {
        for (int ce = 0; ce < T.n_coh; ++ce) {
            const int cn[4] = {T.coh_nodes[ce][0], T.coh_nodes[ce][1], T.coh_nodes[ce][2], T.coh_nodes[ce][3]};
#pragma unroll
            for (int k = 0; k < PPL; ++k) {
                if (lane + 32 * k < npairs) {
                    int i = -1, j = -1;
                    for (int m = 0; m < 4; ++m) {
                        if (cn[m] == pa[k]) i = m;
                        if (cn[m] == pb[k]) j = m;
                    }
                    if (i >= 0 && j >= 0) {
                        const double sgn = ((i < 2) == (j < 2)) ? 1.0 : -1.0;
                        for (int q = 0; q < 2; ++q) {
                            const double* row = sC[w][2 * ce + q];
                            const double wgt = row[0];
                            if (wgt == 0.0) continue;
                            const double v = wgt * sgn * row[1 + (i & 1)] * row[1 + (j & 1)];
                            acc[k][0] += v * row[3];
                            acc[k][1] += v * row[4];
                            acc[k][2] += v * row[5];
                            acc[k][3] += v * row[6];
                        }
                    }
                }
            }
        }
    }
scatter:
    if (SENS) {
        // central difference of wsens . f_e: this pass adds sgn * (its share) / (2 h)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
        if (lane == 0) atomicAdd(&a.sens[sel], a.sgn * part / (2.0 * hstep));
        return;
    }
    if (a.want_K) {
#pragma unroll
        for (int k = 0; k < PPL; ++k) {
            const int p = lane + 32 * k;
            if (p < npairs && slot[k] >= 0) {
                double* d = a.K + 4 * (size_t)slot[k];
                atomicAdd(d + 0, acc[k][0]);
                atomicAdd(d + 1, acc[k][1]);
                atomicAdd(d + 2, acc[k][2]);
                atomicAdd(d + 3, acc[k][3]);
            }
        }
    }
}

__global__ void k_to_fp32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (; i < n / 2; i += stride) {
        const double2 v = reinterpret_cast<const double2*>(a)[i];
        reinterpret_cast<float2*>(b)[i] = make_float2((float)v.x, (float)v.y);
    }
}

template <int W>
void launch_cut_w(int k, const CutArgs& ck, cudaStream_t s) {
    // the two large classes keep at most 4 warps per CTA (48 KB of static shared memory)
    constexpr int WL = W > 4 ? 4 : W;
    const int cblocks = (ck.n_cut + W - 1) / W, lblocks = (ck.n_cut + WL - 1) / WL;
    if (k == 0) k_assemble_cut<5, 1, W><<<cblocks, 32 * W, 0, s>>>(ck);
    else if (k == 1) k_assemble_cut<7, 2, W><<<cblocks, 32 * W, 0, s>>>(ck);
    else if (k == 2) k_assemble_cut<11, 4, WL><<<lblocks, 32 * WL, 0, s>>>(ck);
    else k_assemble_cut<15, 8, WL><<<lblocks, 32 * WL, 0, s>>>(ck);
}

void launch_cut_class(int k, int warps, const CutArgs& ck, cudaStream_t s) {
    if (warps == 2) launch_cut_w<2>(k, ck, s);
    else if (warps == 8) launch_cut_w<8>(k, ck, s);
    else launch_cut_w<4>(k, ck, s);
}


// ---------------------------------------------------------------------------
// Uncut triangles of a structured background grid: edge-centric tiles
// ---------------------------------------------------------------------------
// The background mesh is nx x ny cells of two triangles each (element
// 2 (i + j nx) + t, diagonal alternating with (i + j) % 2), regular node
// (i, j) = i + j (nx + 1).  On such a mesh every off-diagonal block of a
// regular row is a mesh edge: horizontal, vertical, or the diagonal of a
// cell, with at most two triangles on it whose local vertices follow from
// the cells' parities.  Its place in the row is fixed too: the row holds the
// node's grid neighbours (all four axis neighbours; the four diagonal ones
// for even nodes only) in ascending order, then enrichment columns.
// grid_pattern_ok checks that layout on the host before this kernel is used.
//
// A CTA owns a tile of kTileX node columns and TR node rows (3, 4 or 7, picked by
// the autotuner), with the TR + 1 cell rows around them, and runs one thread
// per staged triangle ((TR + 1) x 64) in three phases between two barriers:
//   1. one load per thread of each staged quantity, all in flight at once
//      and addressed by the tile alone: the materials of the staged
//      triangles (-1 marks a cut element), the coordinates (and
//      displacements) of the (TR + 2) x 33 staged nodes, the rows' pointers
//      and the material table;
//   2. one staged triangle per thread: its 6 x 6 stiffness (21 distinct
//      values) into shared memory.  A cell row's triangles are kept t-major
//      (slot 32 t + cell column) at an odd stride of 21 doubles, so the 16
//      lanes of a half-warp reading 16 consecutive cells of one t, or one
//      column each of either t, touch 16 distinct bank pairs;
//   3. per warp two tasks: warps w < TR the horizontal edges and then the
//      diagonal blocks of node row w (zeroing the row's enrichment columns);
//      warps TR .. 2 TR the vertical edges and the cell diagonals of staged
//      cell row w - TR; with WANT_F, the last warp the tile's f_int.
// An edge's block is formed once and stored in both rows (the second as its
// transpose) wherever the tile owns that row; blocks whose triangles are all
// cut are stored as zeros for the cut-element kernel to add to.
constexpr int kTileX = kGridTileX;             // node columns per tile (31)
constexpr int kTileCells = kTileX + 1;         // staged cells per cell row (32)
constexpr int kTileElems = 2 * kTileCells;     // staged triangles per cell row (64)
constexpr int kTileNX = kTileX + 2;            // staged node columns (33)
// Element stiffness in shared memory, kKeStride doubles per triangle: blocks
// (0,1), (0,2), (1,2) row-major at 0, 4, 8 (pair a < b at 4 (a + b - 1));
// diagonal block of vertex v as (k00, k01, k11) at kKeDiag + 3 v.
constexpr int kKeStride = 21;
constexpr int kKeDiag = 12;
constexpr int kKeRow = kTileElems * kKeStride;
// slot of triangle t of staged cell column cc within its cell row
__host__ __device__ constexpr int tile_slot(int cc, int t) { return t * kTileCells + cc; }

struct GridArgs {
    int nx, ny;
    int n_mat;                          // materials (at most kGridMaxMat)
    int strips;                         // tiles across
    int n_tiles;
    // enrichment rows, cleared here for the cut-element kernel to add to:
    // blocks [q_enr, n_blocks) and, with WANT_F, f entries [2 n_reg, 2 n_nodes)
    long long q_enr, n_blocks;
    int n_reg, n_nodes;
    const int* __restrict__ row_ptr;
    const int* __restrict__ emat;       // per element: material, -1 for cut elements
    const double* __restrict__ x;
    const double* __restrict__ y;
    const double* __restrict__ u;
    const double* __restrict__ dmat;
    double* K;
    double* f;
    int want_K;
};

// Corner (di + 2 dj) of local vertex m of triangle t in a cell of parity cp
// ((i + j) % 2): {n00, n10, n11}, {n00, n11, n01} for even cells,
// {n00, n10, n01}, {n10, n11, n01} for odd ones.
__host__ __device__ constexpr int tri_corner(int cp, int t, int m) {
    return cp == 0 ? (t == 0 ? (m == 0 ? 0 : m == 1 ? 1 : 3) : (m == 0 ? 0 : m == 1 ? 3 : 2))
                   : (t == 0 ? (m == 0 ? 0 : m == 1 ? 1 : 2) : (m == 0 ? 1 : m == 1 ? 3 : 2));
}

// Local vertex, in triangle t of a cell of parity cp, of the node at the
// cell's corner (1 - ox, 1 - oy); -1 if the triangle does not touch it.
__host__ __device__ constexpr int sweep_vertex(int cp, int t, int ox, int oy) {
    return tri_corner(cp, t, 0) == (1 - ox) + 2 * (1 - oy) ? 0
         : tri_corner(cp, t, 1) == (1 - ox) + 2 * (1 - oy) ? 1
         : tri_corner(cp, t, 2) == (1 - ox) + 2 * (1 - oy) ? 2 : -1;
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

__device__ __forceinline__ int grid_slot(int row_start, int gi, int gj, int nx, int ny, int d) {
    return row_start + __popc(grid_nbr_mask(gi, gj, nx, ny) & ((1u << d) - 1u));
}

// One 2x2 block as a single 256-bit store (K is a cudaMalloc allocation, so
// every block is 32-byte aligned): half the store requests of two 128-bit ones.
__device__ __forceinline__ void store_block(double* K, int q, double k0, double k1, double k2, double k3) {
    double* dst = K + 4 * (size_t)q;
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(dst), "d"(k0), "d"(k1), "d"(k2), "d"(k3) : "memory");
}

// adds the stored element block at e (4 values, row-major) to k
__device__ __forceinline__ void add_block(const double* e, double k[4]) {
    k[0] += e[0];
    k[1] += e[1];
    k[2] += e[2];
    k[3] += e[3];
}

size_t grid_smem_bytes(bool want_f, int tr) {
    const size_t nodes = (size_t)(tr + 2) * kTileNX;
    return sizeof(double) * ((tr + 1) * (size_t)kKeRow + 2 * nodes + (want_f ? 2 * nodes : 0) + 3 * kGridMaxMat) +
           sizeof(int) * ((tr + 1) * (size_t)kTileElems + tr * (kTileX + 1));
}

// Stiffness of triangle t of staged cell (cc, cr) (material mat >= 0).
__device__ __forceinline__ void tile_element(double* ke, const double* sX, const double* sY, const double* sD,
                                             int mat, int I0, int J0, int cr, int cc, int t) {
    const int cp = (I0 + J0 + cc + cr) & 1;  // parity of cell (I0 - 1 + cc, J0 - 1 + cr)
    double X[3], Y[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const int code = tri_corner(cp, t, m);
        const int k = (cr + (code >> 1)) * kTileNX + cc + (code & 1);
        X[m] = sX[k];
        Y[m] = sY[k];
    }
    const double J = (X[1] - X[0]) * (Y[2] - Y[0]) - (X[2] - X[0]) * (Y[1] - Y[0]);
    const double s = 0.5 / J;
    const double b[3] = {Y[1] - Y[2], Y[2] - Y[0], Y[0] - Y[1]};
    const double c[3] = {X[2] - X[1], X[0] - X[2], X[1] - X[0]};
    const double E0 = s * sD[3 * mat], E1 = s * sD[3 * mat + 1], E2 = s * sD[3 * mat + 2];
    // K_ab = [Xa bb + Wa cb, Ya cb + Wa bb; Va bb + Za cb, Ua cb + Za bb] with
    // X, Y, Z = b (E0, E1, E2), U, V, W = c (E0, E1, E2), E = D / (4 A)
    double Xv[3], Yv[3], Zv[3], Uv[3], Vv[3], Wv[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        Xv[m] = b[m] * E0; Yv[m] = b[m] * E1; Zv[m] = b[m] * E2;
        Uv[m] = c[m] * E0; Vv[m] = c[m] * E1; Wv[m] = c[m] * E2;
    }
#pragma unroll
    for (int pa = 0; pa < 2; ++pa)
#pragma unroll
        for (int pb = pa + 1; pb < 3; ++pb) {
            double* d = ke + 4 * (pa + pb - 1);
            d[0] = Xv[pa] * b[pb] + Wv[pa] * c[pb];
            d[1] = Yv[pa] * c[pb] + Wv[pa] * b[pb];
            d[2] = Vv[pa] * b[pb] + Zv[pa] * c[pb];
            d[3] = Uv[pa] * c[pb] + Zv[pa] * b[pb];
        }
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        double* d = ke + kKeDiag + 3 * m;
        d[0] = Xv[m] * b[m] + Wv[m] * c[m];
        d[1] = Yv[m] * c[m] + Wv[m] * b[m];
        d[2] = Uv[m] * c[m] + Zv[m] * b[m];
    }
}

template <bool WANT_F, int TR>
__global__ void __launch_bounds__((TR + 1) * kTileElems, TR <= 3 ? 4 : (TR <= 4 ? 3 : 2)) k_assemble_grid(GridArgs a) {
    constexpr int kTileThreads = (TR + 1) * kTileElems;  // one staged triangle per thread
    static_assert((TR + 2) * kTileNX <= kTileThreads && TR * (kTileX + 1) <= kTileThreads &&
                  2 * TR + 2 <= kTileThreads / 32, "one staged node and row pointer per thread; warps per task");
    extern __shared__ __align__(16) unsigned char g_tile_smem[];
    constexpr int kNodes = (TR + 2) * kTileNX;
    double* sKe = reinterpret_cast<double*>(g_tile_smem);     // [TR + 1][kTileElems][kKeStride]
    double* sX = sKe + (TR + 1) * kKeRow;                  // [TR + 2][kTileNX]
    double* sY = sX + kNodes;
    double* sU = sY + kNodes;                                  // WANT_F: [TR + 2][2 kTileNX]
    double* sD = sU + (WANT_F ? 2 * kNodes : 0);               // [n_mat][3]: d11, d12, d33
    int* sM = reinterpret_cast<int*>(sD + 3 * kGridMaxMat);   // [TR + 1][kTileElems]
    int* sRp = sM + (TR + 1) * kTileElems;                 // [TR][kTileX + 1]: row pointers
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nx = a.nx, ny = a.ny, NXn = nx + 1;
    const int I0 = (blockIdx.x % a.strips) * kTileX, J0 = (blockIdx.x / a.strips) * TR;
    const int R = min(TR, ny + 1 - J0);  // node rows of this tile
    // this CTA's share of the enrichment rows: cleared (no launch of its own)
    if (a.want_K) {
        const long long n = a.n_blocks - a.q_enr, chunk = (n + a.n_tiles - 1) / a.n_tiles;
        const long long q0 = a.q_enr + blockIdx.x * chunk, q1 = min(q0 + chunk, a.n_blocks);
        for (long long q = q0 + tid; q < q1; q += kTileThreads) store_block(a.K, (int)q, 0.0, 0.0, 0.0, 0.0);
    }
    if (WANT_F) {
        const int n = 2 * (a.n_nodes - a.n_reg), chunk = (n + a.n_tiles - 1) / a.n_tiles;
        const int i0 = 2 * a.n_reg + blockIdx.x * chunk, i1 = min(i0 + chunk, 2 * a.n_nodes);
        for (int i = i0 + tid; i < i1; i += kTileThreads) a.f[i] = 0.0;
    }
    // ---- phase 1: one load per thread of each staged quantity ----
    {
        const int cr = tid / kTileElems, sl = tid % kTileElems;  // slot sl = tile_slot(cc, t)
        const int ci = I0 - 1 + sl % kTileCells, cj = J0 - 1 + cr;
        const int m = (ci >= 0 && ci < nx && cj >= 0 && cj < ny) ? __ldg(&a.emat[2 * (ci + cj * nx) + sl / kTileCells])
                                                                 : -1;
        double xv = 0.0, yv = 0.0, ux = 0.0, uy = 0.0;
        const int gi = I0 - 1 + tid % kTileNX, gj = J0 - 1 + tid / kTileNX;
        const bool in = tid < kNodes && gi >= 0 && gi <= nx && gj >= 0 && gj <= ny;
        if (in) {
            const int node = gi + gj * NXn;
            xv = __ldg(&a.x[node]);
            yv = __ldg(&a.y[node]);
            if (WANT_F) {
                ux = a.u[2 * node];
                uy = a.u[2 * node + 1];
            }
        }
        // row_ptr of tile node (I0 + k, J0 + r); k = kTileX gives the row end of the last one
        const int rk = tid % (kTileX + 1), rr = tid / (kTileX + 1);
        const int rp = rr < R ? __ldg(&a.row_ptr[min(I0 + rk, NXn) + (J0 + rr) * NXn]) : 0;
        const double dm = tid < 3 * a.n_mat ? __ldg(&a.dmat[tid]) : 0.0;
        sM[tid] = m;
        if (tid < kNodes) {
            sX[tid] = xv;
            sY[tid] = yv;
            if (WANT_F) {
                sU[2 * tid] = ux;
                sU[2 * tid + 1] = uy;
            }
        }
        if (rr < TR) sRp[tid] = rp;
        if (tid < 3 * a.n_mat) sD[tid] = dm;
    }
    __syncthreads();
    // ---- phase 2: one staged triangle per thread ----
    {
        const int m = sM[tid], sl = tid % kTileElems;
        if (m >= 0)
            tile_element(sKe + tid * kKeStride, sX, sY, sD, m, I0, J0, tid / kTileElems, sl % kTileCells, sl / kTileCells);
    }
    __syncthreads();
    // ---- phase 3: edges, diagonal blocks, f_int ----
    if (warp < TR) {
        const int r = warp, gj = J0 + r;
        if (r < R) {
            const double* kBelow = sKe + r * kKeRow;        // staged cell row r (global gj - 1)
            const double* kAbove = sKe + (r + 1) * kKeRow;  // staged cell row r + 1 (global gj)
            const int rs = r * (kTileX + 1);
            // horizontal edge A = (gi, gj) - B = (gi + 1, gj), gi = I0 - 1 + lane (tile columns
            // lane - 1 and lane): the top triangle (t = 1, vertices 2, 1) of the cell below,
            // the bottom one (t = 0, vertices 0, 1) of the cell above
            const int gi = I0 - 1 + lane;
            if (a.want_K && gi >= 0 && gi + 1 <= nx) {
                double k[4] = {0.0, 0.0, 0.0, 0.0};
                const int eb = tile_slot(lane, 1), ea = tile_slot(lane, 0);
                if (sM[r * kTileElems + eb] >= 0) {
                    double t[4] = {0.0, 0.0, 0.0, 0.0};
                    add_block(kBelow + eb * kKeStride + 8, t);  // block (1, 2): used transposed
                    k[0] += t[0]; k[1] += t[2]; k[2] += t[1]; k[3] += t[3];
                }
                if (sM[(r + 1) * kTileElems + ea] >= 0) add_block(kAbove + ea * kKeStride + 0, k);
                if (lane >= 1) store_block(a.K, grid_slot(sRp[rs + lane - 1], gi, gj, nx, ny, 5), k[0], k[1], k[2], k[3]);
                if (lane < kTileX) store_block(a.K, grid_slot(sRp[rs + lane], gi + 1, gj, nx, ny, 3), k[0], k[2], k[1], k[3]);
            }
            // diagonal block of node (I0 + lane, gj) over its (at most 8) triangles; zeros in
            // its enrichment columns
            const int gn = I0 + lane;
            if (a.want_K && lane < kTileX && gn <= nx) {
                const int p = (gn + gj) & 1;
                double d0 = 0.0, d1 = 0.0, d2 = 0.0;
#pragma unroll
                for (int oy = 0; oy < 2; ++oy) {
                    const double* kb = oy ? kAbove : kBelow;
#pragma unroll
                    for (int ox = 0; ox < 2; ++ox)
#pragma unroll
                        for (int t = 0; t < 2; ++t) {
                            // staged cell (lane + ox, r + oy), the node at its corner (1 - ox, 1 - oy)
                            const int e = tile_slot(lane + ox, t);
                            const int cp = p ^ ((ox + oy) & 1);
                            const int v = cp ? sweep_vertex(1, t, ox, oy) : sweep_vertex(0, t, ox, oy);
                            if (v < 0 || sM[(r + oy) * kTileElems + e] < 0) continue;
                            const double* dv = kb + e * kKeStride + kKeDiag + 3 * v;
                            d0 += dv[0];
                            d1 += dv[1];
                            d2 += dv[2];
                        }
                }
                const int q0 = sRp[rs + lane], q1 = sRp[rs + lane + 1];
                const unsigned mask = grid_nbr_mask(gn, gj, nx, ny);
                store_block(a.K, q0 + __popc(mask & 15u), d0, d1, d1, d2);
                for (int q = q0 + __popc(mask); q < q1; ++q) store_block(a.K, q, 0.0, 0.0, 0.0, 0.0);
            }
        }
    } else if (warp < TR + TR + 1) {
        // staged cell row s (global gj = J0 - 1 + s) between node rows s - 1 and s
        const int s = warp - TR, gj = J0 - 1 + s;
        const double* kc = sKe + s * kKeRow;
        const bool ownLo = s >= 1 && s - 1 < R, ownHi = s < R;
        if (a.want_K && gj >= 0 && gj < ny) {
            // vertical edge A = (gi, gj) - B = (gi, gj + 1), gi = I0 + lane: in the left cell
            // (parity cl) triangle t = cl with vertices (1, 2) if cl = 0, (0, 1) if cl = 1; in
            // the right cell triangle t = cl with vertices (0, 2)
            const int gi = I0 + lane;
            if (lane < kTileX && gi <= nx) {
                const int cl = (gi - 1 + gj) & 1;
                double k[4] = {0.0, 0.0, 0.0, 0.0};
                const int el = tile_slot(lane, cl), er = tile_slot(lane + 1, cl);
                if (sM[s * kTileElems + el] >= 0) add_block(kc + el * kKeStride + (cl ? 0 : 8), k);
                if (sM[s * kTileElems + er] >= 0) add_block(kc + er * kKeStride + 4, k);
                if (ownLo)
                    store_block(a.K, grid_slot(sRp[(s - 1) * (kTileX + 1) + lane], gi, gj, nx, ny, 7),
                                k[0], k[1], k[2], k[3]);
                if (ownHi)
                    store_block(a.K, grid_slot(sRp[s * (kTileX + 1) + lane], gi, gj + 1, nx, ny, 1),
                                k[0], k[2], k[1], k[3]);
            }
            // diagonal of cell (gc, gj), gc = I0 - 1 + lane, parity cp.  cp = 0: A = (gc, gj),
            // B = (gc + 1, gj + 1), t0 vertices (0, 2), t1 (0, 1).  cp = 1: A = (gc + 1, gj),
            // B = (gc, gj + 1), t0 vertices (1, 2), t1 (0, 2).
            const int gc = I0 - 1 + lane;
            if (gc >= 0 && gc < nx) {
                const int cp = (gc + gj) & 1;
                double k[4] = {0.0, 0.0, 0.0, 0.0};
                const int e0 = tile_slot(lane, 0), e1 = tile_slot(lane, 1);
                if (sM[s * kTileElems + e0] >= 0) add_block(kc + e0 * kKeStride + (cp ? 8 : 4), k);
                if (sM[s * kTileElems + e1] >= 0) add_block(kc + e1 * kKeStride + (cp ? 4 : 0), k);
                const int la = cp ? lane : lane - 1, lb = cp ? lane - 1 : lane;  // tile columns of A, B
                if (ownLo && la >= 0 && la < kTileX)
                    store_block(a.K, grid_slot(sRp[(s - 1) * (kTileX + 1) + la], I0 + la, gj, nx, ny, cp ? 6 : 8),
                                k[0], k[1], k[2], k[3]);
                if (ownHi && lb >= 0 && lb < kTileX)
                    store_block(a.K, grid_slot(sRp[s * (kTileX + 1) + lb], I0 + lb, gj + 1, nx, ny, cp ? 2 : 0),
                                k[0], k[2], k[1], k[3]);
            }
        }
    } else if (WANT_F) {
        // f_int of the tile's nodes, lane = node column
        const int gn = I0 + lane;
        for (int r = 0; r < R; ++r) {
            const int gj = J0 + r;
            if (lane >= kTileX || gn > nx) break;
            const int p = (gn + gj) & 1;
            double fx = 0.0, fy = 0.0;
#pragma unroll
            for (int oy = 0; oy < 2; ++oy) {
                const double* kb = sKe + (r + oy) * kKeRow;
#pragma unroll
                for (int ox = 0; ox < 2; ++ox)
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const int e = tile_slot(lane + ox, t);
                        const int cp = p ^ ((ox + oy) & 1);
                        const int v = cp ? sweep_vertex(1, t, ox, oy) : sweep_vertex(0, t, ox, oy);
                        if (v < 0 || sM[(r + oy) * kTileElems + e] < 0) continue;
                        const double* ke = kb + e * kKeStride;
#pragma unroll
                        for (int m = 0; m < 3; ++m) {
                            double k0, k1, k2, k3;
                            if (m == v) {
                                const double* dv = ke + kKeDiag + 3 * v;
                                k0 = dv[0]; k1 = dv[1]; k2 = dv[1]; k3 = dv[2];
                            } else {
                                const double* eb = ke + 4 * (v + m - 1);
                                k0 = eb[0]; k3 = eb[3];
                                k1 = v < m ? eb[1] : eb[2];
                                k2 = v < m ? eb[2] : eb[1];
                            }
                            const int code = tri_corner(cp, t, m);
                            const int k = (r + oy + (code >> 1)) * kTileNX + lane + ox + (code & 1);
                            const double ux = sU[2 * k], uy = sU[2 * k + 1];
                            fx += k0 * ux + k1 * uy;
                            fy += k2 * ux + k3 * uy;
                        }
                    }
            }
            const int node = gn + gj * NXn;
            a.f[2 * node] = fx;
            a.f[2 * node + 1] = fy;
        }
    }
}

// True when every regular row of the block pattern is laid out as
// k_assemble_grid assumes: the node's grid neighbours (grid_nbr_mask) and
// itself in ascending order, then only enrichment columns.
bool grid_pattern_ok(const HostMesh& hm) {
    const int nx = hm.spec.nx, ny = hm.spec.ny;
    if ((long long)(nx + 1) * (ny + 1) != hm.n_reg) return false;
    for (int gj = 0; gj <= ny; ++gj)
        for (int gi = 0; gi <= nx; ++gi) {
            const int i = gi + gj * (nx + 1);
            const unsigned mask = grid_nbr_mask(gi, gj, nx, ny);
            int q = hm.row_ptr[i];
            for (int d = 0; d < 9; ++d) {
                if (!(mask & (1u << d))) continue;
                const int j = (gi + d % 3 - 1) + (gj + d / 3 - 1) * (nx + 1);
                if (q >= hm.row_ptr[i + 1] || hm.col[q] != j) return false;
                ++q;
            }
            for (; q < hm.row_ptr[i + 1]; ++q)
                if (hm.col[q] < hm.n_reg) return false;
        }
    return true;
}

// Lifts k_assemble_grid's dynamic shared-memory limit, once per device and
// outside any graph capture (called when a context is created).
void grid_prepare() {
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev]) return;
    cudaFuncSetAttribute(k_assemble_grid<false, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(false, 3));
    cudaFuncSetAttribute(k_assemble_grid<true, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(true, 3));
    cudaFuncSetAttribute(k_assemble_grid<false, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(false, 4));
    cudaFuncSetAttribute(k_assemble_grid<true, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(true, 4));
    cudaFuncSetAttribute(k_assemble_grid<false, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(false, 7));
    cudaFuncSetAttribute(k_assemble_grid<true, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grid_smem_bytes(true, 7));
    if (dev >= 0 && dev < 64) done[dev] = true;
}

void launch_grid(const Ctx& c, const double* U, bool want_f, bool want_K, cudaStream_t s) {
    GridArgs ga;
    ga.nx = c.hm.spec.nx;
    ga.ny = c.hm.spec.ny;
    ga.n_mat = (int)c.hm.spec.materials.size();
    ga.row_ptr = c.row_ptr;
    ga.emat = c.grid_emat;
    ga.x = c.x;
    ga.y = c.y;
    ga.u = U;
    ga.dmat = c.dmat;
    ga.K = c.K;
    ga.f = c.F;
    ga.want_K = want_K;
    ga.strips = (ga.nx + 1 + kTileX - 1) / kTileX;
    const int tr = c.tuning.grid_rows == 3 ? 3 : c.tuning.grid_rows == 4 ? 4 : 7;
    const int tiles = ga.strips * ((ga.ny + 1 + tr - 1) / tr);
    ga.n_tiles = tiles;
    ga.q_enr = c.hm.row_ptr[c.n_reg];
    ga.n_blocks = c.n_blocks;
    ga.n_reg = c.n_reg;
    ga.n_nodes = c.n_nodes;
    const int threads = (tr + 1) * kTileElems;
    grid_prepare();
    if (tr == 3) {
        if (want_f) k_assemble_grid<true, 3><<<tiles, threads, grid_smem_bytes(true, 3), s>>>(ga);
        else k_assemble_grid<false, 3><<<tiles, threads, grid_smem_bytes(false, 3), s>>>(ga);
    } else if (tr == 4) {
        if (want_f) k_assemble_grid<true, 4><<<tiles, threads, grid_smem_bytes(true, 4), s>>>(ga);
        else k_assemble_grid<false, 4><<<tiles, threads, grid_smem_bytes(false, 4), s>>>(ga);
    } else {
        if (want_f) k_assemble_grid<true, 7><<<tiles, threads, grid_smem_bytes(true, 7), s>>>(ga);
        else k_assemble_grid<false, 7><<<tiles, threads, grid_smem_bytes(false, 7), s>>>(ga);
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

// Shape-sensitivity passes of the cut-element kernel (one per size class).
void launch_cut_sens(const Ctx& c, const CutArgs& ca, cudaStream_t s) {
    for (int k = 0; k < kCutClasses; ++k) {
        const int n = c.cut_class_off[k + 1] - c.cut_class_off[k];
        if (n == 0) continue;
        CutArgs ck = ca;
        ck.n_cut = n;
        ck.first = c.cut_class_off[k];
        const int blocks = (n + 3) / 4;
        if (k == 0) k_assemble_cut<5, 1, 4, true><<<blocks, 128, 0, s>>>(ck);
        else if (k == 1) k_assemble_cut<7, 2, 4, true><<<blocks, 128, 0, s>>>(ck);
        else if (k == 2) k_assemble_cut<11, 4, 4, true><<<blocks, 128, 0, s>>>(ck);
        else k_assemble_cut<15, 8, 4, true><<<blocks, 128, 0, s>>>(ck);
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

CutArgs cut_args(const Ctx& c, const double* U, double dt, bool want_f, bool want_K) {
    CutArgs ca;
    ca.n_cut = c.n_cut;
    ca.first = 0;
    ca.cut_nodes = c.cut_nodes;
    ca.cut_tmpl = c.cut_tmpl;
    ca.cut_child_mat = c.cut_child_mat;
    ca.cut_coh_qp0 = c.cut_coh_qp0;
    ca.cut_slot_ptr = c.cut_slot_ptr;
    ca.cut_slot = c.cut_slot;
    ca.x = c.x;
    ca.y = c.y;
    ca.u = U;
    ca.dmat = c.dmat;
    ca.isv_c = c.isv_c;
    ca.isv_t = c.isv_t;
    ca.rows = c.cut_rows;
    ca.row_off = c.cut_row_off;
    ca.coh = c.coh;
    ca.dt = dt;
    ca.K = c.K;
    ca.f = c.F;
    ca.want_K = want_K;
    ca.want_f = want_f;
    return ca;
}

void launch_cut_points(const Ctx& c, cudaStream_t s) {
    if (c.n_cut_pts > 0) {
        CutPointArgs pa;
        pa.n_pts = c.n_cut_pts;
        pa.pts = reinterpret_cast<const int4*>(c.cut_pts);
        pa.x = c.x;
        pa.y = c.y;
        pa.dmat = c.dmat;
        pa.rows = c.cut_rows;
        k_cut_points<<<(c.n_cut_pts + 255) / 256, 256, 0, s>>>(pa);
    }
}

void launch_cut_classes(const Ctx& c, const CutArgs& ca, cudaStream_t s) {
    for (int k = 0; k < kCutClasses; ++k) {
        const int n = c.cut_class_off[k + 1] - c.cut_class_off[k];
        if (n == 0) continue;
        CutArgs ck = ca;
        ck.n_cut = n;
        ck.first = c.cut_class_off[k];
        launch_cut_class(k, c.tuning.cut_warps, ck, s);
    }
}

void launch_cut_all(const Ctx& c, const CutArgs& ca, cudaStream_t s) {
    launch_cut_points(c, s);
    launch_cut_classes(c, ca, s);
}

int launch_assemble(Ctx& c, const double* U, double dt, bool want_f, bool want_K, cudaStream_t s) {
    // nothing to clear: the triangle kernel writes every value of K
    const RowArgs ra = row_args(c, U, want_f, want_K);
    // the cut elements' quadrature rows depend on the coordinates only: they
    // are formed on the second stream beside the triangle kernel.  That one is
    // launched first, so its CTAs are dispatched first and the row kernel's
    // fill the SMs its last wave leaves free.
    const bool fork = c.n_cut_pts > 0;
    if (fork) PG_CUDA(cudaEventRecord(c.fork_ev, s));
    if (c.timing) cudaEventRecord(c.ea0, s);
    launch_tri(c, ra, want_f, s);
    PG_CUDA(cudaGetLastError());
    if (fork) {
        PG_CUDA(cudaStreamWaitEvent(c.aux, c.fork_ev, 0));
        launch_cut_points(c, c.aux);
        PG_CUDA(cudaEventRecord(c.join_ev, c.aux));
    }
    if (c.timing) cudaEventRecord(c.ea1, s);
    if (fork) PG_CUDA(cudaStreamWaitEvent(s, c.join_ev, 0));
    if (c.n_cut > 0) {
        launch_cut_classes(c, cut_args(c, U, dt, want_f, want_K), s);
        PG_CUDA(cudaGetLastError());
    }
    if (c.timing) cudaEventRecord(c.ea2, s);
    return PG_OK;
}

// Times every launch shape of the two assembly kernels on this mesh (L2
// flushed before each launch, `reps` launches each, device events) and keeps
// the fastest of each kernel in c.tuning.  ms_tri: tile 32/64 x one CTA per
// tile / persistent (4 values), ms_cut: 2/4/8 warps per CTA (3 values).  K is
// left undefined (the cut kernel ran repeatedly): the next solve reassembles.
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
    if (c.grid_emat) {
        // the structured-grid kernel at both tile heights; ms_tri[4] reports the faster
        c.tuning.tri_grid = 1;
        float ms_grid = 0.f;
        for (int tr : {3, 4, 7}) {
            c.tuning.grid_rows = tr;
            const RowArgs ra = row_args(c, c.U, false, true);
            const float ms = timed([&] { launch_tri(c, ra, false, s); });
            if (ms_grid == 0.f || ms < ms_grid) ms_grid = ms;
            if (ms < best_tri) {
                best_tri = ms;
                best.tri_grid = 1;
                best.grid_rows = tr;
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
        if (c.n_cut > 0) {
            const CutArgs ca = cut_args(c, c.U, 1.0, false, true);
            ms = timed([&] { launch_cut_all(c, ca, s); });
        }
        if (ms_cut) ms_cut[k] = ms;
        if (ms < best_cut) {
            best_cut = ms;
            best.cut_warps = warps[k];
        }
    }
    c.tuning = best;
    c.assembled = false;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(flush);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

int launch_to_fp32(Ctx& c, cudaStream_t s) {
    const size_t n = 4 * (size_t)c.n_blocks;
    k_to_fp32<<<148 * 8, 256, 0, s>>>(c.K, c.Kf, n);
    PG_CUDA(cudaGetLastError());
    return PG_OK;
}

}  // namespace pgb
