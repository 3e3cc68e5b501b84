/*
 * CPU ORACLE -- test infrastructure only.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load this; the product never does.
 *
 * Plain-C FP64 restatement of the reference's element integration and
 * assembly for the IGFEM path, written to follow the reference's per-
 * quadrature-point algorithm step by step (not the B200 kernels' algebra):
 *
 *   Assembler::assemble_elem_linear / _nonlinear   PIGFEM4.6.1/src/Assembler.cpp:94-185, 305-528
 *   Mesh::store_shape_functions                    src/Mesh.cpp:1443-1605
 *     child q_point -> child ShapeFunctions -> global point -> parent
 *     inverse_map -> parent ShapeFunctions -> enrichment functions taken
 *     from the child's functions at the matching nodes
 *   Elem::transform_gradients                      src/elem.cpp:112-136
 *   Tri3 q_point (order 3) / inverse_map           src/tri3.cpp:93-141, 200-217
 *   Quad4 q_point / shapes                         src/quad4.cpp:108-148
 *   Polygon q_point / shapes (order mismatch kept) src/Polygon.cpp:51-228
 *   CohesiveElem ShapeFunctions / rotation         src/CohesiveElem.cpp:145-238, src/CohEdge2.cpp:60-160
 *   ProblemUtilities::SmallStrainKFast             src/Utilities.cpp:196-296
 *   ProblemUtilities::SmallStrainFast / IntForce   src/Utilities.cpp:300-408
 *   ProblemUtilities::cohesiveDeltaFast/KFast/Int  src/Utilities.cpp:465-531
 *   LinearElasticIsotropicMaterial::computeLinearDmat / computeStress  src/material_lei.cpp:52-97, 232-261
 *   OPCohesiveMaterial::Constitutive               src/Material_OPCohesive.cpp:38-388
 *   OPCohesiveNUMaterial::getDeltaEff              src/Material_OPCohesiveNU.cpp:45-63
 *
 * Input: a fully explicit enriched mesh (coordinates, connectivity, per cut
 * element its enrichment nodes, children and cohesive sub-elements in local
 * numbering).  Output: the DOF-level matrix in CSR (node-major DOFs
 * 2*node+d), the internal force vector, and the trial cohesive state.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846264338327950
#define MAXN 15

typedef struct {
    int n_nodes;
    const double* xy;           /* 2*n_nodes */
    int n_elem;
    const int32_t* conn;        /* 3*n_elem */
    const int32_t* elem_mat;    /* material of an uncut element */
    const int32_t* is_cut;      /* per element 0/1 */
    /* per element (CSR-like, only cut elements have entries) */
    const int32_t* enr_ptr;     /* n_elem+1 */
    const int32_t* enr;         /* global node id of each enrichment slot */
    const int32_t* child_ptr;   /* n_elem+1, children of element e */
    const int32_t* child_nodes_ptr; /* n_children_total+1 */
    const int32_t* child_nodes; /* local node ids */
    const int32_t* child_mat;   /* per child */
    const int32_t* coh_ptr;     /* n_elem+1 */
    const int32_t* coh_nodes;   /* 4 local ids per cohesive sub-element */
    int n_mat;
    const double* mat_E;
    const double* mat_nu;
    int plane_strain;
    /* cohesive law: 0 = Ortiz-Pandolfi (sigma_c, delta_c, beta, viscosity), 1 = bilinear (sigma_c, G_c, K_p, beta) */
    int coh_law;
    double coh_p[5];
} orc_mesh;

/* ---------------- constitutive ---------------- */
static void dmat(const orc_mesh* m, int mat, double D[3][3]) {
    double E = m->mat_E[mat], nu = m->mat_nu[mat];
    memset(D, 0, sizeof(double) * 9);
    if (m->plane_strain) {
        double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
        D[0][0] = coef * (1.0 - nu); D[0][1] = coef * (nu);
        D[1][0] = coef * (nu);       D[1][1] = coef * (1.0 - nu);
        D[2][2] = coef * (1.0 - 2.0 * nu) / 2.0;
    } else {
        double coef = E / (1.0 - nu * nu);
        D[0][0] = coef; D[0][1] = coef * nu;
        D[1][0] = coef * nu; D[1][1] = coef;
        D[2][2] = coef * (1.0 - nu) / 2.0;
    }
}

/* K(2n x 2n) = B^T D B exploiting B's zeros, the SmallStrainKFast dim-2 loop */
static void small_strain_K(int n, const double dN[][2], const double D[3][3], double* K /* (2n)^2 */) {
    int ndof = 2 * n;
    for (int row = 0; row < ndof; ++row) {
        int is = row % 2, in = row / 2;
        double p0, p1, p2;
        if (is == 0) {
            p0 = dN[in][0] * D[0][0] + dN[in][1] * D[2][0];
            p1 = dN[in][0] * D[0][1] + dN[in][1] * D[2][1];
            p2 = dN[in][0] * D[0][2] + dN[in][1] * D[2][2];
        } else {
            p0 = dN[in][1] * D[1][0] + dN[in][0] * D[2][0];
            p1 = dN[in][1] * D[1][1] + dN[in][0] * D[2][1];
            p2 = dN[in][1] * D[1][2] + dN[in][0] * D[2][2];
        }
        for (int col = 0; col < ndof; ++col) {
            int js = col % 2, jn = col / 2;
            K[row * ndof + col] = js == 0 ? p0 * dN[jn][0] + p2 * dN[jn][1] : p1 * dN[jn][1] + p2 * dN[jn][0];
        }
    }
}

/* OP law, returns traction t (ttn), tangent Dc, updated trial delta_max */
static void op_law(const orc_mesh* m, double dt, double dmax, double delta[2], double t[2], double Dc[2][2], double* dmax_out) {
    const double sc = m->coh_p[0], dc = m->coh_p[1], beta2 = m->coh_p[2] * m->coh_p[2], visc = m->coh_p[3];
    double norm = delta[0] * delta[0] + delta[1] * delta[1];
    if (norm < 1e-40) { delta[0] = 1e-20; delta[1] = 1e-20; }
    double de = pow(delta[1], 2);
    de += beta2 * pow(delta[0], 2);
    de = sqrt(de);
    double T, dT;
    *dmax_out = dmax;
    if (de >= dmax || de < 0.0) {
        T = sc * (de / dc) * exp(1.0 - de / dc) + visc / sc * (de - dmax) / dt / dc;
        dT = (sc / dc) * (1.0 - de / dc) * exp(1.0 - de / dc) + visc / sc / dt / dc;
        *dmax_out = de;
    } else {
        double Tm = sc * (dmax / dc) * exp(1.0 - dmax / dc);
        T = Tm * (de / dmax);
        dT = Tm / dmax;
    }
    double br[2] = {beta2 * delta[0], beta2 * delta[1]};
    br[1] += (1.0 - beta2) * delta[1];
    for (int i = 0; i < 2; ++i) t[i] = (T / de) * br[i];
    double dd[2] = {beta2 * delta[0] / de, delta[1] / de};
    for (int i = 0; i < 2; ++i)
        for (int k = 0; k < 2; ++k)
            Dc[i][k] = br[i] * (dT * de - T) * (dd[k] / pow(de, 2)) +
                       (T / de) * (beta2 * (i == k) + (1.0 - beta2) * (i == 1) * (k == 1));
}

/* bilinear penalty law (sigma_c, G_c, K_p, beta, eta) with normal compression penalty and the
   viscous traction eta (delta_eff - delta_max) / dt while loading */
static void bilinear_law(const orc_mesh* m, double dt, double dmax, double delta[2], double t[2], double Dc[2][2], double* dmax_out) {
    const double sc = m->coh_p[0], Gc = m->coh_p[1], Kp = m->coh_p[2], beta2 = m->coh_p[3] * m->coh_p[3];
    const double d0 = sc / Kp, df = 2.0 * Gc / sc;
    double norm = delta[0] * delta[0] + delta[1] * delta[1];
    if (norm < 1e-40) { delta[0] = 1e-20; delta[1] = 1e-20; }
    double dn = delta[1] > 0.0 ? delta[1] : 0.0;
    double de = sqrt(dn * dn + beta2 * delta[0] * delta[0]) + 1e-300;
    double T, dT;
    *dmax_out = dmax;
    #define ENV(dd, T_, dT_) do { if ((dd) <= d0) { T_ = Kp * (dd); dT_ = Kp; } \
        else if ((dd) < df) { T_ = sc * (df - (dd)) / (df - d0); dT_ = -sc / (df - d0); } else { T_ = 0.0; dT_ = 0.0; } } while (0)
    if (de >= dmax) { ENV(de, T, dT); T += m->coh_p[4] * (de - dmax) / dt; dT += m->coh_p[4] / dt; *dmax_out = de; }
    else { double Tm, dTm; ENV(dmax, Tm, dTm); (void)dTm; T = Tm * (de / dmax); dT = Tm / dmax; }
    #undef ENV
    double s = T / de, a = dT * de - T, de2 = de * de;
    double br0 = beta2 * delta[0], br1 = dn, dd0 = beta2 * delta[0] / de, dd1 = dn / de;
    t[0] = s * br0;
    Dc[0][0] = br0 * a * (dd0 / de2) + s * beta2;
    if (delta[1] >= 0.0) {
        t[1] = s * br1;
        Dc[0][1] = br0 * a * (dd1 / de2);
        Dc[1][0] = br1 * a * (dd0 / de2);
        Dc[1][1] = br1 * a * (dd1 / de2) + s;
    } else {
        t[1] = Kp * delta[1];
        Dc[0][1] = 0.0; Dc[1][0] = 0.0; Dc[1][1] = Kp;
    }
}

/* ---------------- reference elements ---------------- */
static const double TRI3_Q[4][3] = {{0.333333333333333333333333333333333, 0.333333333333333333333333333333333, -0.281250000000000000000000000000000},
                                    {0.200000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665},
                                    {0.200000000000000000000000000000000, 0.600000000000000000000000000000000, 0.260416666666666666666666666666665},
                                    {0.600000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665}};
static const double TRI5_Q[7][3] = {{0.33333333333333, 0.33333333333333, 0.112500000000000},
                                    {0.47014206410511, 0.47014206410511, 0.066197076394255},
                                    {0.47014206410511, 0.05971587178977, 0.066197076394255},
                                    {0.05971587178977, 0.47014206410511, 0.066197076394255},
                                    {0.10128650732346, 0.10128650732346, 0.062969590272415},
                                    {0.10128650732346, 0.79742698535309, 0.062969590272415},
                                    {0.79742698535309, 0.10128650732346, 0.062969590272415}};
static const double G2 = 0.57735026918962576450914878050196;

static void poly_triangulate(int nn, double r, double s, double px[], double py[]) {
    for (int n = 0; n < nn; ++n) {
        px[n] = cos(2.0 * ORC_PI * (n + 1) / nn);
        py[n] = sin(2.0 * ORC_PI * (n + 1) / nn);
    }
    px[nn] = r; py[nn] = s;
}

static void poly_shape(int nn, double r, double s, double N[], double dN[][2]) {
    double px[8], py[8], A[8], dA[8][2], al[8], dal[8][2];
    poly_triangulate(nn, r, s, px, py);
    for (int n = 0; n < nn; ++n) {
        int t0 = nn, t1 = n, t2 = (n + 1 == nn) ? 0 : n + 1;
        double p0x = px[t0], p0y = py[t0], p1x = px[t1], p1y = py[t1], p2x = px[t2], p2y = py[t2];
        A[n + 1] = 0.5 * ((p1x * p2y - p1y * p2x) - (p0x * p2y - p0y * p2x) + (p0x * p1y - p0y * p1x));
        dA[n + 1][0] = 0.5 * (p2y - p1y);
        dA[n + 1][1] = 0.5 * (p1x - p2x);
    }
    A[0] = A[nn]; dA[0][0] = dA[nn][0]; dA[0][1] = dA[nn][1];
    double sa = 0.0, sd0 = 0.0, sd1 = 0.0;
    for (int n = 0; n < nn; ++n) {
        al[n] = 1.0 / (A[n] * A[n + 1]);
        dal[n][0] = -1.0 * al[n] * (dA[n][0] / A[n] + dA[n + 1][0] / A[n + 1]);
        dal[n][1] = -1.0 * al[n] * (dA[n][1] / A[n] + dA[n + 1][1] / A[n + 1]);
        sa += al[n]; sd0 += dal[n][0]; sd1 += dal[n][1];
    }
    for (int n = 0; n < nn; ++n) {
        N[n] = al[n] / sa;
        dN[n][0] = (dal[n][0] - N[n] * sd0) / sa;
        dN[n][1] = (dal[n][1] - N[n] * sd1) / sa;
    }
}

/* quadrature point qp of a child with nc nodes: reference coords and weight */
static int child_nq(int nc) { return nc == 3 ? 4 : nc == 4 ? 4 : 4 * nc; }
static void child_qp(int nc, int qp, double* r, double* s, double* w) {
    if (nc == 3) { *r = TRI3_Q[qp][0]; *s = TRI3_Q[qp][1]; *w = TRI3_Q[qp][2]; return; }
    if (nc == 4) {
        double g[2] = {-G2, G2};
        *r = g[qp % 2]; *s = g[qp / 2]; *w = 1.0 * 1.0; return;
    }
    /* polygon: n*4 points from the order-5 triangle rule (qp%7, triangle qp/7) */
    int tq = qp % 7, tri = qp / 7;
    double tr = TRI5_Q[tq][0], ts = TRI5_Q[tq][1], tw = TRI5_Q[tq][2];
    double tN[3] = {1.0 - tr - ts, tr, ts};
    double tdN[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
    double px[8], py[8];
    poly_triangulate(nc, 0.0, 0.0, px, py);
    int ids[3] = {nc, tri, (tri + 1 == nc) ? 0 : tri + 1};
    double J0[2][2] = {{0, 0}, {0, 0}};
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j)
            for (int n = 0; n < 3; ++n) J0[i][j] += (i == 0 ? px[ids[n]] : py[ids[n]]) * tdN[n][j];
    *w = (J0[0][0] * J0[1][1] - J0[0][1] * J0[1][0]) * tw;
    *r = 0.0; *s = 0.0;
    for (int n = 0; n < 3; ++n) { *r += tN[n] * px[ids[n]]; *s += tN[n] * py[ids[n]]; }
}

static void child_shape(int nc, double r, double s, double N[], double dN[][2]) {
    if (nc == 3) {
        N[0] = 1.0 - r - s; N[1] = r; N[2] = s;
        dN[0][0] = -1.0; dN[0][1] = -1.0; dN[1][0] = 1.0; dN[1][1] = 0.0; dN[2][0] = 0.0; dN[2][1] = 1.0;
    } else if (nc == 4) {
        N[0] = 0.25 * (1.0 - r) * (1.0 - s); N[1] = 0.25 * (1.0 + r) * (1.0 - s);
        N[2] = 0.25 * (1.0 + r) * (1.0 + s); N[3] = 0.25 * (1.0 - r) * (1.0 + s);
        dN[0][0] = -0.25 * (1.0 - s); dN[0][1] = -0.25 * (1.0 - r);
        dN[1][0] = 0.25 * (1.0 - s);  dN[1][1] = -0.25 * (1.0 + r);
        dN[2][0] = 0.25 * (1.0 + s);  dN[2][1] = 0.25 * (1.0 + r);
        dN[3][0] = -0.25 * (1.0 + s); dN[3][1] = 0.25 * (1.0 - r);
    } else {
        poly_shape(nc, r, s, N, dN);
    }
}

/* Elem::transform_gradients: Jac(a,i) = sum_n dNdr[n][a] x_n(i); J = det; dNdx = Jinv dNdr */
static double transform(int nn, const double X[][2], const double dNr[][2], double dNx[][2]) {
    double Jac[2][2] = {{0, 0}, {0, 0}};
    for (int a = 0; a < 2; ++a)
        for (int i = 0; i < 2; ++i)
            for (int n = 0; n < nn; ++n) Jac[a][i] += dNr[n][a] * X[n][i];
    double J = Jac[0][0] * Jac[1][1] - Jac[0][1] * Jac[1][0];
    double inv[2][2] = {{Jac[1][1], -1.0 * Jac[0][1]}, {-1.0 * Jac[1][0], Jac[0][0]}};
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) inv[a][b] *= (1.0 / J);
    for (int n = 0; n < nn; ++n) {
        dNx[n][0] = inv[0][0] * dNr[n][0] + inv[0][1] * dNr[n][1];
        dNx[n][1] = inv[1][0] * dNr[n][0] + inv[1][1] * dNr[n][1];
    }
    return J;
}

/* Tri3::inverse_map */
static void tri3_inverse_map(const double c[3][2], double gx, double gy, double* r, double* s) {
    double A = 0.5 * (c[0][0] * (c[1][1] - c[2][1]) + c[1][0] * (c[2][1] - c[0][1]) + c[2][0] * (c[0][1] - c[1][1]));
    if (A < 0.0) A = -1.0 * A;
    *r = (1.0 / (2.0 * A)) * ((c[2][1] - c[0][1]) * (gx - c[0][0]) - (c[2][0] - c[0][0]) * (gy - c[0][1]));
    *s = (1.0 / (2.0 * A)) * (-1.0 * (c[1][1] - c[0][1]) * (gx - c[0][0]) + (c[1][0] - c[0][0]) * (gy - c[0][1]));
}

/* ---------------- DOF-level CSR accumulation ---------------- */
typedef struct {
    int n;
    int32_t* rp;
    int32_t* col;
    double* val;
} csr_t;

static int cmp_int(const void* a, const void* b) { int x = *(const int*)a, y = *(const int*)b; return (x > y) - (x < y); }

static void csr_add(csr_t* K, int i, int j, double v) {
    int lo = K->rp[i], hi = K->rp[i + 1] - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (K->col[mid] == j) { K->val[mid] += v; return; }
        if (K->col[mid] < j) lo = mid + 1; else hi = mid - 1;
    }
}

/* element local node list (3 parent nodes then enrichment slots) */
static int elem_nodes(const orc_mesh* m, int e, int L[MAXN]) {
    for (int v = 0; v < 3; ++v) L[v] = m->conn[3 * e + v];
    int n = 3;
    if (m->is_cut[e])
        for (int k = m->enr_ptr[e]; k < m->enr_ptr[e + 1]; ++k) L[n++] = m->enr[k];
    return n;
}

/* Pattern: returns nnz; rp has 2n+1 entries, col must hold nnz (call with col=NULL to count) */
int orc_pattern(const orc_mesh* m, int32_t* rp, int32_t* col) {
    int ndof = 2 * m->n_nodes;
    /* node adjacency lists */
    int* cnt = (int*)calloc((size_t)m->n_nodes + 1, sizeof(int));
    for (int e = 0; e < m->n_elem; ++e) {
        int L[MAXN], n = elem_nodes(m, e, L);
        for (int a = 0; a < n; ++a) cnt[L[a] + 1] += n;
    }
    for (int i = 0; i < m->n_nodes; ++i) cnt[i + 1] += cnt[i];
    int* adj = (int*)malloc(sizeof(int) * (size_t)(cnt[m->n_nodes] + 1));
    int* fill = (int*)malloc(sizeof(int) * (size_t)m->n_nodes);
    for (int i = 0; i < m->n_nodes; ++i) fill[i] = cnt[i];
    for (int e = 0; e < m->n_elem; ++e) {
        int L[MAXN], n = elem_nodes(m, e, L);
        for (int a = 0; a < n; ++a)
            for (int b = 0; b < n; ++b) adj[fill[L[a]]++] = L[b];
    }
    int nnz = 0;
    if (rp) rp[0] = 0;
    for (int i = 0; i < m->n_nodes; ++i) {
        int* s = adj + cnt[i];
        int k = fill[i] - cnt[i];
        qsort(s, (size_t)k, sizeof(int), cmp_int);
        int u = 0;
        for (int t = 0; t < k; ++t)
            if (u == 0 || s[t] != s[u - 1]) s[u++] = s[t];
        for (int d = 0; d < 2; ++d) {
            if (col)
                for (int t = 0; t < u; ++t) { col[nnz + 2 * t] = 2 * s[t]; col[nnz + 2 * t + 1] = 2 * s[t] + 1; }
            nnz += 2 * u;
            if (rp) rp[2 * i + d + 1] = nnz;
        }
    }
    (void)ndof;
    free(cnt); free(adj); free(fill);
    return nnz;
}

/*
 * Assembles K (into the CSR pattern from orc_pattern, values zeroed here)
 * and/or f_int at displacement u (node-major, 2*n_nodes), writing trial
 * cohesive state isv_t from committed isv_c (one value per cohesive qp in
 * element / sub-element / qp order).  want_K/want_f select the outputs.
 * Returns 0, or a positive code on a geometry error (negative Jacobian,
 * bad inverse map), the conditions the reference stops on.
 */
int orc_assemble(const orc_mesh* m, const int32_t* rp, const int32_t* col, double* val, const double* u, double dt,
                 const double* isv_c, double* isv_t, double* f, int want_K, int want_f) {
    csr_t K = {2 * m->n_nodes, (int32_t*)rp, (int32_t*)col, val};
    if (want_K) memset(val, 0, sizeof(double) * (size_t)rp[2 * m->n_nodes]);
    if (want_f) memset(f, 0, sizeof(double) * (size_t)(2 * m->n_nodes));
    int coh_qp = 0;
    double* Kel = (double*)malloc(sizeof(double) * (2 * MAXN) * (2 * MAXN));
    double* Kt = (double*)malloc(sizeof(double) * (2 * MAXN) * (2 * MAXN));
    double Pel[2 * MAXN];
    for (int e = 0; e < m->n_elem; ++e) {
        int L[MAXN], nl = elem_nodes(m, e, L);
        int nd = 2 * nl;
        double X[MAXN][2], ue[2 * MAXN];
        for (int a = 0; a < nl; ++a) {
            X[a][0] = m->xy[2 * L[a]]; X[a][1] = m->xy[2 * L[a] + 1];
            ue[2 * a] = u ? u[2 * L[a]] : 0.0; ue[2 * a + 1] = u ? u[2 * L[a] + 1] : 0.0;
        }
        memset(Kel, 0, sizeof(double) * nd * nd);
        memset(Pel, 0, sizeof(Pel));
        double parent[3][2] = {{X[0][0], X[0][1]}, {X[1][0], X[1][1]}, {X[2][0], X[2][1]}};
        if (!m->is_cut[e]) {
            double D[3][3];
            dmat(m, m->elem_mat[e], D);
            for (int qp = 0; qp < 4; ++qp) {
                double N[3], dNr[3][2], dNx[3][2];
                child_shape(3, TRI3_Q[qp][0], TRI3_Q[qp][1], N, dNr);
                double J = transform(3, parent, dNr, dNx);
                if (J < -1e-16) { free(Kel); free(Kt); return 1; }
                double wgt = J * TRI3_Q[qp][2];
                small_strain_K(3, (const double(*)[2])dNx, D, Kt);
                /* K_el.AXPY(wgt, K_temp) is cblas_daxpy, which returns at once
                   for a zero weight (DenseMatrix.h:424-431) */
                if (wgt != 0.0)
                    for (int i = 0; i < 36; ++i) Kel[i] += wgt * Kt[i];
            }
        } else {
            for (int c = m->child_ptr[e]; c < m->child_ptr[e + 1]; ++c) {
                int nc = m->child_nodes_ptr[c + 1] - m->child_nodes_ptr[c];
                const int32_t* cn = m->child_nodes + m->child_nodes_ptr[c];
                double D[3][3];
                dmat(m, m->child_mat[c], D);
                double CX[8][2];
                for (int k = 0; k < nc; ++k) { CX[k][0] = X[cn[k]][0]; CX[k][1] = X[cn[k]][1]; }
                for (int qp = 0; qp < child_nq(nc); ++qp) {
                    double r, s, W, cN[8], cdNr[8][2], cdNx[8][2];
                    child_qp(nc, qp, &r, &s, &W);
                    child_shape(nc, r, s, cN, cdNr);
                    double J = transform(nc, (const double(*)[2])CX, (const double(*)[2])cdNr, cdNx);
                    if (J < 0.0) { free(Kel); free(Kt); return 2; }
                    double gx = 0.0, gy = 0.0;
                    for (int k = 0; k < nc; ++k) { gx += CX[k][0] * cN[k]; gy += CX[k][1] * cN[k]; }
                    double pr, ps;
                    tri3_inverse_map(parent, gx, gy, &pr, &ps);
                    double pN[3], pdNr[3][2], pdNx[3][2];
                    child_shape(3, pr, ps, pN, pdNr);
                    transform(3, parent, pdNr, pdNx);
                    double g2x = 0.0, g2y = 0.0;
                    for (int k = 0; k < 3; ++k) { g2x += parent[k][0] * pN[k]; g2y += parent[k][1] * pN[k]; }
                    if (sqrt(pow(g2x - gx, 2) + pow(g2y - gy, 2)) > 1e-9) { free(Kel); free(Kt); return 3; }
                    double G[MAXN][2];
                    memset(G, 0, sizeof(G));
                    for (int k = 0; k < 3; ++k) { G[k][0] = pdNx[k][0]; G[k][1] = pdNx[k][1]; }
                    for (int en = 3; en < nl; ++en)
                        for (int k = 0; k < nc; ++k)
                            if (cn[k] == en) { G[en][0] = cdNx[k][0]; G[en][1] = cdNx[k][1]; break; }
                    small_strain_K(nl, (const double(*)[2])G, D, Kt);
                    double wgt = J * W;
                    if (wgt != 0.0) /* zero-weight points are skipped, as cblas_daxpy does */
                        for (int i = 0; i < nd * nd; ++i) Kel[i] += wgt * Kt[i];
                }
            }
        }
        /* bulk internal force: linear elastic, f = (sum wgt B^T D B) u_e */
        if (want_f)
            for (int i = 0; i < nd; ++i) {
                double sacc = 0.0;
                for (int j = 0; j < nd; ++j) sacc += Kel[i * nd + j] * ue[j];
                Pel[i] += sacc;
            }
        /* cohesive sub-elements */
        if (m->is_cut[e])
            for (int ce = m->coh_ptr[e]; ce < m->coh_ptr[e + 1]; ++ce) {
                const int32_t* hn = m->coh_nodes + 4 * ce;
                /* rotation from the lower-surface nodes (CohesiveElem::compute_rotation) */
                double Jac[2] = {0.0, 0.0};
                double pg[2] = {-0.5, 0.5};
                for (int n = 0; n < 2; ++n)
                    for (int i = 0; i < 2; ++i) Jac[i] += pg[n] * X[hn[n]][i];
                double nrm[2] = {-Jac[1], Jac[0]};
                double mag = sqrt(Jac[0] * Jac[0] + Jac[1] * Jac[1]);
                double dA = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
                double R[2][2] = {{Jac[0] / mag, Jac[1] / mag}, {nrm[0] / dA, nrm[1] / dA}};
                double cu[8];
                for (int n = 0; n < 4; ++n) { cu[2 * n] = ue[2 * hn[n]]; cu[2 * n + 1] = ue[2 * hn[n] + 1]; }
                double Kc[8][8], Pc[8];
                memset(Kc, 0, sizeof(Kc)); memset(Pc, 0, sizeof(Pc));
                for (int qp = 0; qp < 2; ++qp) {
                    double xi = qp == 0 ? -G2 : G2;
                    double Nn[2] = {0.5 * (1.0 - xi), 0.5 * (1 + xi)};
                    double dg[2] = {0.0, 0.0};
                    for (int d = 0; d < 2; ++d)
                        for (int n = 0; n < 2; ++n) dg[d] += Nn[n] * (cu[(n + 2) * 2 + d] - cu[n * 2 + d]);
                    double dl[2] = {R[0][0] * dg[0] + R[0][1] * dg[1], R[1][0] * dg[0] + R[1][1] * dg[1]};
                    double t[2], Dc[2][2], dnew;
                    double dmax = isv_c ? isv_c[coh_qp] : 0.0;
                    if (m->coh_law == 0) op_law(m, dt, dmax, dl, t, Dc, &dnew);
                    else bilinear_law(m, dt, dmax, dl, t, Dc, &dnew);
                    if (isv_t) isv_t[coh_qp] = dnew;
                    ++coh_qp;
                    double RDR[2][2], tR[2];
                    for (int i = 0; i < 2; ++i)
                        for (int j = 0; j < 2; ++j) {
                            double sacc = 0.0;
                            for (int a = 0; a < 2; ++a)
                                for (int b = 0; b < 2; ++b) sacc += R[a][i] * Dc[a][b] * R[b][j];
                            RDR[i][j] = sacc;
                        }
                    for (int i = 0; i < 2; ++i) tR[i] = R[0][i] * t[0] + R[1][i] * t[1];
                    double wgt = dA * 1.0;
                    if (wgt == 0.0) continue; /* K_coh.AXPY / daxpy skip a zero weight */
                    for (int n1 = 0; n1 < 2; ++n1)
                        for (int n2 = 0; n2 < 2; ++n2)
                            for (int d1 = 0; d1 < 2; ++d1)
                                for (int d2 = 0; d2 < 2; ++d2) {
                                    double v = Nn[n1] * Nn[n2] * RDR[d1][d2];
                                    Kc[n1 * 2 + d1][n2 * 2 + d2] += wgt * v;
                                    Kc[(n1 + 2) * 2 + d1][n2 * 2 + d2] += wgt * -v;
                                    Kc[n1 * 2 + d1][(n2 + 2) * 2 + d2] += wgt * -v;
                                    Kc[(n1 + 2) * 2 + d1][(n2 + 2) * 2 + d2] += wgt * v;
                                }
                    for (int n = 0; n < 2; ++n)
                        for (int d = 0; d < 2; ++d) {
                            double v = Nn[n] * tR[d];
                            Pc[n * 2 + d] += wgt * -v;
                            Pc[(n + 2) * 2 + d] += wgt * v;
                        }
                }
                for (int n1 = 0; n1 < 4; ++n1)
                    for (int d1 = 0; d1 < 2; ++d1) {
                        int row = hn[n1] * 2 + d1;
                        for (int n2 = 0; n2 < 4; ++n2)
                            for (int d2 = 0; d2 < 2; ++d2) Kel[row * nd + hn[n2] * 2 + d2] += Kc[n1 * 2 + d1][n2 * 2 + d2];
                        Pel[row] += Pc[n1 * 2 + d1];
                    }
            }
        if (want_K)
            for (int a = 0; a < nl; ++a)
                for (int da = 0; da < 2; ++da)
                    for (int b = 0; b < nl; ++b)
                        for (int db = 0; db < 2; ++db)
                            csr_add(&K, 2 * L[a] + da, 2 * L[b] + db, Kel[(2 * a + da) * nd + 2 * b + db]);
        if (want_f)
            for (int a = 0; a < nl; ++a)
                for (int da = 0; da < 2; ++da) f[2 * L[a] + da] += Pel[2 * a + da];
    }
    free(Kel); free(Kt);
    return 0;
}

/* Element-level entry for tests: K_e of a single uncut triangle (6x6). */
void orc_tri3_K(const double xy[6], double E, double nu, int plane_strain, double Ke[36]) {
    orc_mesh m;
    memset(&m, 0, sizeof(m));
    m.mat_E = &E; m.mat_nu = &nu; m.plane_strain = plane_strain; m.n_mat = 1;
    double D[3][3];
    dmat(&m, 0, D);
    double X[3][2] = {{xy[0], xy[1]}, {xy[2], xy[3]}, {xy[4], xy[5]}};
    double Kt[36];
    memset(Ke, 0, sizeof(double) * 36);
    for (int qp = 0; qp < 4; ++qp) {
        double N[3], dNr[3][2], dNx[3][2];
        child_shape(3, TRI3_Q[qp][0], TRI3_Q[qp][1], N, dNr);
        double J = transform(3, X, dNr, dNx);
        small_strain_K(3, (const double(*)[2])dNx, D, Kt);
        for (int i = 0; i < 36; ++i) Ke[i] += J * TRI3_Q[qp][2] * Kt[i];
    }
}

/* Cohesive law point evaluation for tests. */
void orc_cohesive_law(int law, const double p[5], double dt, double dmax, double delta_in[2], double t[2], double Dc[4],
                      double* dmax_out) {
    orc_mesh m;
    memset(&m, 0, sizeof(m));
    m.coh_law = law;
    for (int i = 0; i < 5; ++i) m.coh_p[i] = p[i];
    double D2[2][2];
    if (law == 0) op_law(&m, dt, dmax, delta_in, t, D2, dmax_out);
    else bilinear_law(&m, dt, dmax, delta_in, t, D2, dmax_out);
    Dc[0] = D2[0][0]; Dc[1] = D2[0][1]; Dc[2] = D2[1][0]; Dc[3] = D2[1][1];
}
