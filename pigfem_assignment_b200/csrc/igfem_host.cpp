// Host-side IGFEM preprocessing (see igfem_host.h for the reference
// functions each step restates).
#include "igfem_host.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <set>
#include <sstream>
#include <utility>

namespace pgb {

namespace {

constexpr double kPi = 3.14159265358979323846264338327950;  // common.h PI
const int kEdgeNodes[3][2] = {{0, 1}, {1, 2}, {2, 0}};        // Tri3::e_n_map (tri3.cpp:21-26)

// ---------------------------------------------------------------------------
// Cut templates: the branches of Tri3::detection (tri3.cpp:287-541), stored as
// data.  Ids 0..9 are the perfectly bonded cases, 10..22 the cohesive ones.
//   single(k):   one inclusion, node k on its own side
//   two(k):      two inclusions, node k alone in its inclusion
//   three_m(k):  three regions, node k in the matrix
//   three:       every node in a different inclusion
// ---------------------------------------------------------------------------
std::vector<CutTemplate> make_templates() {
    std::vector<CutTemplate> t;
    auto add = [&](int nce, bool coh, std::vector<int> ce, std::vector<int> einc,
                   std::vector<std::vector<int>> ch, std::vector<int> cmat,
                   std::vector<std::vector<int>> cohs) {
        CutTemplate c{};
        c.n_cut_edges = nce;
        c.n_enr = coh ? 2 * nce : nce;
        for (int i = 0; i < nce; ++i) { c.cut_edge[i] = ce[i]; c.enr_inc_node[i] = einc[i]; }
        c.n_child = (int)ch.size();
        for (int i = 0; i < c.n_child; ++i) {
            c.child_n[i] = (int)ch[i].size();
            for (int j = 0; j < c.child_n[i]; ++j) c.child_nodes[i][j] = ch[i][j];
            c.child_mat_node[i] = cmat[i];
        }
        c.n_coh = (int)cohs.size();
        for (int i = 0; i < c.n_coh; ++i)
            for (int j = 0; j < 4; ++j) c.coh_nodes[i][j] = cohs[i][j];
        t.push_back(c);
    };
    const int M = -1;  // the element's own (matrix) material / "largest value" inclusion
    // ---- perfectly bonded ----
    add(2, false, {0, 2}, {M, M}, {{0, 3, 4}, {1, 2, 4, 3}}, {0, 1}, {});                 // 0 single(0)
    add(2, false, {0, 1}, {M, M}, {{1, 4, 3}, {0, 3, 4, 2}}, {1, 2}, {});                 // 1 single(1)
    add(2, false, {1, 2}, {M, M}, {{2, 4, 3}, {0, 1, 3, 4}}, {2, 0}, {});                 // 2 single(2)
    add(4, false, {2, 0, 2, 0}, {0, 0, 1, 1}, {{0, 4, 3}, {4, 6, 5, 3}, {1, 2, 5, 6}}, {0, M, 1}, {});  // 3 two(0)
    add(4, false, {0, 1, 0, 1}, {1, 1, 2, 2}, {{1, 4, 3}, {4, 6, 5, 3}, {2, 0, 5, 6}}, {1, M, 2}, {});  // 4 two(1)
    add(4, false, {1, 2, 1, 2}, {2, 2, 0, 0}, {{2, 4, 3}, {4, 6, 5, 3}, {0, 1, 5, 6}}, {2, M, 0}, {});  // 5 two(2)
    add(4, false, {1, 0, 2, 1}, {1, 1, 2, 2}, {{1, 3, 4}, {0, 4, 3, 6, 5}, {2, 5, 6}}, {1, M, 2}, {});  // 6 three_m(0)
    add(4, false, {2, 1, 0, 2}, {2, 2, 0, 0}, {{2, 3, 4}, {1, 4, 3, 6, 5}, {0, 5, 6}}, {2, M, 0}, {});  // 7 three_m(1)
    add(4, false, {0, 2, 1, 0}, {0, 0, 1, 1}, {{0, 3, 4}, {2, 4, 3, 6, 5}, {1, 5, 6}}, {0, M, 1}, {});  // 8 three_m(2)
    add(6, false, {0, 2, 2, 1, 1, 0}, {0, 0, 2, 2, 1, 1},
        {{0, 3, 4}, {2, 5, 6}, {1, 7, 8}, {8, 7, 6, 5, 4, 3}}, {0, 2, 1, M}, {});           // 9 three
    // ---- cohesive ----
    // single(k), node k in the matrix (n_k < n_other)
    add(2, true, {2, 0}, {M, M}, {{0, 4, 3}, {1, 2, 5, 6}}, {0, 1}, {{3, 4, 5, 6}});      // 10
    add(2, true, {0, 1}, {M, M}, {{1, 4, 3}, {2, 0, 5, 6}}, {1, 0}, {{3, 4, 5, 6}});      // 11
    add(2, true, {1, 2}, {M, M}, {{2, 4, 3}, {0, 1, 5, 6}}, {2, 0}, {{3, 4, 5, 6}});      // 12
    // single(k), node k in the inclusion
    add(2, true, {2, 0}, {M, M}, {{0, 6, 5}, {1, 2, 3, 4}}, {0, 1}, {{4, 3, 6, 5}});      // 13
    add(2, true, {0, 1}, {M, M}, {{1, 6, 5}, {2, 0, 3, 4}}, {1, 0}, {{4, 3, 6, 5}});      // 14
    add(2, true, {1, 2}, {M, M}, {{2, 6, 5}, {0, 1, 3, 4}}, {2, 0}, {{4, 3, 6, 5}});      // 15
    add(4, true, {2, 0, 2, 0}, {0, 0, 1, 1}, {{0, 8, 7}, {4, 6, 5, 3}, {1, 2, 9, 10}}, {0, M, 1},
        {{4, 3, 8, 7}, {5, 6, 9, 10}});                                                    // 16 two(0)
    add(4, true, {0, 1, 0, 1}, {1, 1, 2, 2}, {{1, 8, 7}, {4, 6, 5, 3}, {2, 0, 9, 10}}, {1, M, 2},
        {{4, 3, 8, 7}, {5, 6, 9, 10}});                                                    // 17 two(1)
    add(4, true, {1, 2, 1, 2}, {2, 2, 0, 0}, {{2, 8, 7}, {4, 6, 5, 3}, {0, 1, 9, 10}}, {2, M, 0},
        {{4, 3, 8, 7}, {5, 6, 9, 10}});                                                    // 18 two(2)
    add(4, true, {1, 0, 2, 1}, {1, 1, 2, 2}, {{1, 7, 8}, {0, 4, 3, 6, 5}, {2, 9, 10}}, {1, M, 2},
        {{3, 4, 7, 8}, {5, 6, 9, 10}});                                                    // 19 three_m(0)
    add(4, true, {2, 1, 0, 2}, {2, 2, 0, 0}, {{2, 7, 8}, {1, 4, 3, 6, 5}, {0, 9, 10}}, {2, M, 0},
        {{3, 4, 7, 8}, {5, 6, 9, 10}});                                                    // 20 three_m(1)
    add(4, true, {0, 2, 1, 0}, {0, 0, 1, 1}, {{0, 7, 8}, {2, 4, 3, 6, 5}, {1, 9, 10}}, {0, M, 1},
        {{3, 4, 7, 8}, {5, 6, 9, 10}});                                                    // 21 three_m(2)
    add(6, true, {0, 2, 2, 1, 1, 0}, {0, 0, 2, 2, 1, 1},
        {{0, 9, 10}, {2, 11, 12}, {1, 13, 14}, {8, 7, 6, 5, 4, 3}}, {0, 2, 1, M},
        {{3, 4, 9, 10}, {5, 6, 11, 12}, {7, 8, 13, 14}});                                  // 22 three
    return t;
}

const std::vector<CutTemplate>& templates() {
    static const std::vector<CutTemplate> t = make_templates();
    return t;
}

// Template choice from the three nodal detection values (-1 = matrix),
// following the case analysis of Tri3::detection.  Returns -1 if uncut.
int choose_template(const int d[3], bool cohesive, std::string& err) {
    int vals[3] = {d[0], d[1], d[2]};
    std::sort(vals, vals + 3);
    const int n_unique = 1 + (vals[1] != vals[0]) + (vals[2] != vals[1]);
    if (n_unique == 1) return -1;
    const bool e01 = d[0] == d[1], e02 = d[0] == d[2], e12 = d[1] == d[2];
    const int base = cohesive ? 10 : 0;
    if (n_unique == 2) {
        int k;  // the separate node
        if (e12) k = 0;
        else if (e02) k = 1;
        else if (e01) k = 2;
        else { err = "triangle with one node separated in an unknown manner"; return -2; }
        if (vals[0] < 0) {
            if (!cohesive) return k;
            const int other = (k + 1) % 3;
            return d[k] < d[other] ? 10 + k : 13 + k;
        }
        return base + (cohesive ? 6 : 3) + k;
    }
    // three unique values
    if (vals[0] < 0) {
        int k = d[0] < 0 ? 0 : (d[1] < 0 ? 1 : 2);
        return base + (cohesive ? 9 : 6) + k;
    }
    return cohesive ? 22 : 9;
}

// ---------------------------------------------------------------------------
// Quadrature tables of the child (integration) elements.
// ---------------------------------------------------------------------------
// Tri3 order-3 rule (tri3.cpp:107-115) and order-5 rule (tri3.cpp:130-140).
const double kTri3Q[4][3] = {{0.333333333333333333333333333333333, 0.333333333333333333333333333333333, -0.281250000000000000000000000000000},
                             {0.200000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665},
                             {0.200000000000000000000000000000000, 0.600000000000000000000000000000000, 0.260416666666666666666666666666665},
                             {0.600000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665}};
const double kTri5Q[7][3] = {{0.33333333333333, 0.33333333333333, 0.112500000000000},
                             {0.47014206410511, 0.47014206410511, 0.066197076394255},
                             {0.47014206410511, 0.05971587178977, 0.066197076394255},
                             {0.05971587178977, 0.47014206410511, 0.066197076394255},
                             {0.10128650732346, 0.10128650732346, 0.062969590272415},
                             {0.10128650732346, 0.79742698535309, 0.062969590272415},
                             {0.79742698535309, 0.10128650732346, 0.062969590272415}};
const double kGauss2 = 0.57735026918962576450914878050196;  // edge2.cpp:122-123

// Wachspress-type polygon functions on the regular n-gon inscribed in the unit
// circle with vertex k at angle 2*pi*(k+1)/n (Polygon.cpp:51-228).
void polygon_shape(int nn, double r, double s, std::vector<double>& N, std::vector<double>& dN) {
    std::vector<double> px(nn + 1), py(nn + 1);
    for (int k = 0; k < nn; ++k) {
        px[k] = std::cos(2.0 * kPi * (k + 1) / nn);
        py[k] = std::sin(2.0 * kPi * (k + 1) / nn);
    }
    px[nn] = r;
    py[nn] = s;
    // sub-triangle k = (point, vertex k, vertex k+1)
    std::vector<double> A(nn + 1), dAx(nn + 1), dAy(nn + 1);
    for (int k = 0; k < nn; ++k) {
        const int a = nn, b = k, c = (k + 1) % nn;
        const double x0 = px[a], y0 = py[a], x1 = px[b], y1 = py[b], x2 = px[c], y2 = py[c];
        A[k + 1] = 0.5 * ((x1 * y2 - y1 * x2) - (x0 * y2 - y0 * x2) + (x0 * y1 - y0 * x1));
        dAx[k + 1] = 0.5 * (y2 - y1);
        dAy[k + 1] = 0.5 * (x1 - x2);
    }
    A[0] = A[nn]; dAx[0] = dAx[nn]; dAy[0] = dAy[nn];
    std::vector<double> al(nn), dax(nn), day(nn);
    double sa = 0, sdx = 0, sdy = 0;
    for (int k = 0; k < nn; ++k) {
        al[k] = 1.0 / (A[k] * A[k + 1]);
        dax[k] = -al[k] * (dAx[k] / A[k] + dAx[k + 1] / A[k + 1]);
        day[k] = -al[k] * (dAy[k] / A[k] + dAy[k + 1] / A[k + 1]);
        sa += al[k]; sdx += dax[k]; sdy += day[k];
    }
    N.resize(nn);
    dN.resize(2 * nn);
    for (int k = 0; k < nn; ++k) {
        N[k] = al[k] / sa;
        dN[2 * k] = (dax[k] - N[k] * sdx) / sa;
        dN[2 * k + 1] = (day[k] - N[k] * sdy) / sa;
    }
}

std::vector<ChildQuadrature> make_child_quadrature() {
    std::vector<ChildQuadrature> q(kNumChildTypes);
    {   // Tri3
        ChildQuadrature& c = q[kChildTri3];
        c.nq = 4; c.nn = 3;
        for (int i = 0; i < 4; ++i) {
            const double r = kTri3Q[i][0], s = kTri3Q[i][1];
            c.w.push_back(kTri3Q[i][2]);
            c.N.insert(c.N.end(), {1.0 - r - s, r, s});
            c.dN.insert(c.dN.end(), {-1.0, -1.0, 1.0, 0.0, 0.0, 1.0});
        }
    }
    {   // Quad4: 2x2 Gauss, point qp = (g[qp%2], g[qp/2]) (quad4.cpp:108-126)
        ChildQuadrature& c = q[kChildQuad4];
        c.nq = 4; c.nn = 4;
        const double g[2] = {-kGauss2, kGauss2};
        for (int i = 0; i < 4; ++i) {
            const double r = g[i % 2], s = g[i / 2];
            c.w.push_back(1.0);
            c.N.insert(c.N.end(), {0.25 * (1.0 - r) * (1.0 - s), 0.25 * (1.0 + r) * (1.0 - s),
                                   0.25 * (1.0 + r) * (1.0 + s), 0.25 * (1.0 - r) * (1.0 + s)});
            c.dN.insert(c.dN.end(), {-0.25 * (1.0 - s), -0.25 * (1.0 - r), 0.25 * (1.0 - s), -0.25 * (1.0 + r),
                                     0.25 * (1.0 + s), 0.25 * (1.0 + r), -0.25 * (1.0 + s), 0.25 * (1.0 - r)});
        }
    }
    // Polygons: the reference counts n*4 points (n_q_points with the default
    // order 3) but fetches them from the order-5 triangle rule (q_point's
    // default order 5): point qp lies in sub-triangle qp/7 at rule entry qp%7.
    // That mismatch is reproduced as is.
    for (int nn : {5, 6}) {
        ChildQuadrature& c = q[nn == 5 ? kChildPoly5 : kChildPoly6];
        c.nn = nn;
        c.nq = nn * 4;
        std::vector<double> px(nn + 1), py(nn + 1);
        for (int k = 0; k < nn; ++k) {
            px[k] = std::cos(2.0 * kPi * (k + 1) / nn);
            py[k] = std::sin(2.0 * kPi * (k + 1) / nn);
        }
        px[nn] = 0.0; py[nn] = 0.0;
        for (int qp = 0; qp < c.nq; ++qp) {
            const int tri = qp / 7, tq = qp % 7;
            const int ia = nn, ib = tri, ic = (tri + 1) % nn;
            const double tr = kTri5Q[tq][0], ts = kTri5Q[tq][1], tw = kTri5Q[tq][2];
            const double tN[3] = {1.0 - tr - ts, tr, ts};
            const double pTx[3] = {px[ia], px[ib], px[ic]}, pTy[3] = {py[ia], py[ib], py[ic]};
            // J0[i][j] = sum_n pT[n][i] * dN_tri[n][j], dN_tri = {{-1,-1},{1,0},{0,1}}
            const double J00 = -pTx[0] + pTx[1], J01 = -pTx[0] + pTx[2];
            const double J10 = -pTy[0] + pTy[1], J11 = -pTy[0] + pTy[2];
            c.w.push_back((J00 * J11 - J01 * J10) * tw);
            double r = 0, s = 0;
            for (int k = 0; k < 3; ++k) { r += tN[k] * pTx[k]; s += tN[k] * pTy[k]; }
            std::vector<double> N, dN;
            polygon_shape(nn, r, s, N, dN);
            c.N.insert(c.N.end(), N.begin(), N.end());
            c.dN.insert(c.dN.end(), dN.begin(), dN.end());
        }
    }
    return q;
}

// Point on the edge p0 -> p1 where the circle is crossed: the root in [0, 1]
// of f(a) = |p0 + a (p1 - p0) - c|^2 / r^2 - 1, the level set the reference
// brackets and solves iteratively (Inclusion.cpp:32-128,
// InclusionCircle.cpp:248-287).  Here the quadratic is solved in closed form
// (cancellation-free root pair) and polished with two Newton steps on f.
bool circle_edge_root(double x0, double y0, double x1, double y1, const Inclusion& inc, double& alpha) {
    auto f = [&](double a) {
        const double gx = (x0 + a * (x1 - x0) - inc.cx) / inc.r;
        const double gy = (y0 + a * (y1 - y0) - inc.cy) / inc.r;
        return gx * gx + gy * gy - 1.0;
    };
    if (f(0.0) * f(1.0) >= 0.0) return false;
    const double dx = (x1 - x0) / inc.r, dy = (y1 - y0) / inc.r;
    const double ex = (x0 - inc.cx) / inc.r, ey = (y0 - inc.cy) / inc.r;
    const double qa = dx * dx + dy * dy;
    const double qb = 2.0 * (ex * dx + ey * dy);
    const double qc = ex * ex + ey * ey - 1.0;
    const double disc = std::max(qb * qb - 4.0 * qa * qc, 0.0);
    const double q = -0.5 * (qb + std::copysign(std::sqrt(disc), qb));
    double r1 = q / qa, r2 = (q != 0.0) ? qc / q : r1;
    double a = (r1 >= 0.0 && r1 <= 1.0) ? r1 : r2;
    if (!(a >= 0.0 && a <= 1.0)) a = std::min(std::max(a, 0.0), 1.0);
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

}  // namespace

const CutTemplate& cut_template(int id) { return templates()[id]; }
int n_cut_templates() { return (int)templates().size(); }

const ChildQuadrature& child_quadrature(int type) {
    static const std::vector<ChildQuadrature> q = make_child_quadrature();
    return q[type];
}

std::string build_mesh(const RveSpec& spec, HostMesh& m) {
    std::ostringstream err;
    m = HostMesh();
    m.spec = spec;
    const int nx = spec.nx, ny = spec.ny;
    if (nx < 1 || ny < 1) return "mesh needs at least one element in each direction";
    if ((long long)(nx + 1) * (ny + 1) > (1ll << 28)) return "mesh too large";
    if (spec.materials.empty() || spec.matrix_mat < 0 || spec.matrix_mat >= (int)spec.materials.size())
        return "invalid matrix material";
    for (const auto& inc : spec.inclusions)
        if (inc.r <= 0.0 || inc.mat < 0 || inc.mat >= (int)spec.materials.size()) return "invalid inclusion";

    // ---- structured TRI3 mesh (Mesh.cpp:250-405) ----
    const double hx = (spec.x1 - spec.x0) / nx, hy = (spec.y1 - spec.y0) / ny;
    m.n_reg = (nx + 1) * (ny + 1);
    m.x.resize(m.n_reg);
    m.y.resize(m.n_reg);
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            m.x[i + j * (nx + 1)] = spec.x0 + i * hx;
            m.y[i + j * (nx + 1)] = spec.y0 + j * hy;
        }
    m.n_elem = 2 * nx * ny;
    m.grids.push_back({nx, ny, 0, 0, m.n_reg});
    m.conn.resize(3 * (size_t)m.n_elem);
    {
        size_t e = 0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int n00 = i + j * (nx + 1), n10 = n00 + 1, n01 = n00 + (nx + 1), n11 = n01 + 1;
                const int* pat;
                int a[6];
                if ((i + j) % 2 == 0) { int t[6] = {n00, n10, n11, n00, n11, n01}; std::copy(t, t + 6, a); }
                else { int t[6] = {n00, n10, n01, n10, n11, n01}; std::copy(t, t + 6, a); }
                pat = a;
                for (int k = 0; k < 6; ++k) m.conn[e * 3 + k] = pat[k];
                e += 2;
            }
    }
    m.elem_mat.assign(m.n_elem, spec.matrix_mat);

    // the first element (in element order) a node belongs to: the node-moving
    // rule takes its edge length from it (Mesh::generate_node_elem lists a
    // node's elements in element order).  A node's cells in increasing index
    // order, each cell's two triangles in order.
    auto first_elem = [&](int n) {
        const int gi = n % (nx + 1), gj = n / (nx + 1);
        const int cells[4][2] = {{gi - 1, gj - 1}, {gi, gj - 1}, {gi - 1, gj}, {gi, gj}};
        for (const auto& cl : cells) {
            if (cl[0] < 0 || cl[0] >= nx || cl[1] < 0 || cl[1] >= ny) continue;
            for (int t = 0; t < 2; ++t) {
                const int e = 2 * (cl[0] + cl[1] * nx) + t;
                for (int v = 0; v < 3; ++v)
                    if (m.conn[3 * (size_t)e + v] == n) return e;
            }
        }
        return -1;
    };

    // ---- node detection with the node-moving rule (Mesh.cpp:2838-2918) ----
    // A node is tested against the inclusions in descending order, and only
    // those whose bounding box holds it get past the first test.  So the
    // inclusions are binned by bounding box on a uniform grid of cells about
    // one diameter wide, and a node walks its cell's list (ascending, read
    // backwards): the same inclusions in the same order as a scan over all.
    const int ninc = (int)spec.inclusions.size();
    double dmax = 0.0;
    for (const auto& inc : spec.inclusions) dmax = std::max(dmax, 2.0 * inc.r);
    const double W = spec.x1 - spec.x0, H = spec.y1 - spec.y0;
    const int nbx = dmax > 0.0 ? std::max(1, std::min(256, (int)(W / dmax))) : 1;
    const int nby = dmax > 0.0 ? std::max(1, std::min(256, (int)(H / dmax))) : 1;
    const double bsx = W / nbx, bsy = H / nby;
    // floor((v - v0) / bs) clamped to the grid: monotonic in v, so a point
    // inside a bounding box lands in one of the box's cells
    auto bin_of = [](double v, double v0, double bs, int nb) {
        const double f = std::floor((v - v0) / bs);
        return f < 0.0 ? 0 : (f >= nb ? nb - 1 : (int)f);
    };
    std::vector<std::vector<int>> bins((size_t)nbx * nby);
    for (int j = 0; j < ninc; ++j) {
        const Inclusion& inc = spec.inclusions[j];
        const int i0 = bin_of(inc.cx - inc.r, spec.x0, bsx, nbx), i1 = bin_of(inc.cx + inc.r, spec.x0, bsx, nbx);
        const int j0 = bin_of(inc.cy - inc.r, spec.y0, bsy, nby), j1 = bin_of(inc.cy + inc.r, spec.y0, bsy, nby);
        for (int bj = j0; bj <= j1; ++bj)
            for (int bi = i0; bi <= i1; ++bi) bins[(size_t)bj * nbx + bi].push_back(j);
    }
    m.node_detect.assign(m.n_reg, -1);
    for (int n = 0; n < m.n_reg; ++n) {
        int moved = 0;
        int result = -1;
        const std::vector<int>* list =
            &bins[(size_t)bin_of(m.y[n], spec.y0, bsy, nby) * nbx + bin_of(m.x[n], spec.x0, bsx, nbx)];
        for (int li = (int)list->size() - 1; li >= 0; --li) {
            const int j = (*list)[li];
            const Inclusion& inc = spec.inclusions[j];
            const double px = m.x[n], py = m.y[n];
            if (!(inc.cx - inc.r <= px && inc.cy - inc.r <= py && px <= inc.cx + inc.r && py <= inc.cy + inc.r)) continue;
            const double dx = px - inc.cx, dy = py - inc.cy;
            const double val = (std::sqrt(dx * dx + dy * dy) - inc.r) / inc.r;
            const double eps = 1e-12;
            if (val > eps) continue;
            if (val < -eps) { result = j; break; }
            // on the interface: move 5% of an element edge along the outward normal
            if (moved >= 5) { err << "unable to move node " << n << " off an inclusion surface"; return err.str(); }
            const double nrm = std::sqrt(dx * dx + dy * dy);
            const double nxn = dx / nrm, nyn = dy / nrm;
            const int e0 = first_elem(n);
            int other = m.conn[3 * e0 + 0];
            if (other == n) other = m.conn[3 * e0 + 1];
            const double ox = m.x[other], oy = m.y[other];
            const double dist = 0.05 * std::sqrt((px - ox) * (px - ox) + (py - oy) * (py - oy) + 0.0);
            m.x[n] = px + dist * nxn;
            m.y[n] = py + dist * nyn;
            ++moved;
            ++m.n_moved;
            // restart the scan over the inclusions, from the moved node's cell
            list = &bins[(size_t)bin_of(m.y[n], spec.y0, bsy, nby) * nbx + bin_of(m.x[n], spec.x0, bsx, nbx)];
            li = (int)list->size();
        }
        m.node_detect[n] = result;
    }

    // ---- element detection (Mesh.cpp:2922-3027, tri3.cpp:287-541) ----
    m.elem_cut.assign(m.n_elem, -1);
    for (int e = 0; e < m.n_elem; ++e) {
        int d[3];
        for (int v = 0; v < 3; ++v) d[v] = m.node_detect[m.conn[3 * e + v]];
        std::string terr;
        const int t = choose_template(d, spec.cohesive, terr);
        if (t == -2) { err << "element " << e << ": " << terr; return err.str(); }
        if (t < 0) {
            if (d[0] != -1) m.elem_mat[e] = spec.inclusions[d[0]].mat;
            continue;
        }
        const CutTemplate& T = templates()[t];
        m.elem_cut[e] = m.n_cut++;
        m.cut_elem.push_back(e);
        m.cut_tmpl.push_back(t);
        for (int c = 0; c < kMaxChildren; ++c) {
            int mat = -1;
            if (c < T.n_child) {
                const int k = T.child_mat_node[c];
                mat = (k < 0 || d[k] < 0) ? m.elem_mat[e] : spec.inclusions[d[k]].mat;
            }
            m.cut_child_mat.push_back(mat);
        }
        for (int c = 0; c < kMaxCoh; ++c) m.cut_coh_mat.push_back(c < T.n_coh ? 0 : -1);
    }

    // ---- enrichment nodes (Mesh.cpp:3064-3202, 3600-3660) ----
    // unique (edge, inclusion) pairs in the reference's std::set order: the
    // keys sorted lexicographically and made unique
    using EdgeKey = std::pair<std::pair<int, int>, int>;
    std::vector<int> slot_inc(m.n_cut * 6, -1);
    std::vector<EdgeKey> cut_edges;
    for (int c = 0; c < m.n_cut; ++c) {
        const int e = m.cut_elem[c];
        const CutTemplate& T = templates()[m.cut_tmpl[c]];
        int d[3], dmax = -1;
        for (int v = 0; v < 3; ++v) { d[v] = m.node_detect[m.conn[3 * e + v]]; dmax = std::max(dmax, d[v]); }
        for (int s = 0; s < T.n_cut_edges; ++s) {
            const int inc = T.enr_inc_node[s] < 0 ? dmax : d[T.enr_inc_node[s]];
            slot_inc[c * 6 + s] = inc;
            int a = m.conn[3 * e + kEdgeNodes[T.cut_edge[s]][0]], b = m.conn[3 * e + kEdgeNodes[T.cut_edge[s]][1]];
            if (a > b) std::swap(a, b);
            cut_edges.push_back({{a, b}, inc});
        }
    }
    std::sort(cut_edges.begin(), cut_edges.end());
    cut_edges.erase(std::unique(cut_edges.begin(), cut_edges.end()), cut_edges.end());
    m.n_enr_initial = (int)cut_edges.size();
    m.n_enr = spec.cohesive ? 2 * m.n_enr_initial : m.n_enr_initial;
    m.x.resize(m.n_reg + m.n_enr);
    m.y.resize(m.n_reg + m.n_enr);
    m.enr_edge.resize(2 * m.n_enr);
    m.enr_inc.resize(m.n_enr);
    {
        int k = 0;
        for (const auto& ce : cut_edges) {
            const int a = ce.first.first, b = ce.first.second, inc = ce.second;
            double alpha;
            if (!circle_edge_root(m.x[a], m.y[a], m.x[b], m.y[b], spec.inclusions[inc], alpha)) {
                err << "no valid intersection between nodes " << a << " and " << b;
                return err.str();
            }
            double ex = m.x[a] + alpha * (m.x[b] - m.x[a]);
            double ey = m.y[a] + alpha * (m.y[b] - m.y[a]);
            // An interface that passes through a mesh node to within rounding
            // (a node the moving rule misses because its bounding-box test
            // rounds it out, Mesh.cpp:2850) puts the intersection on the node:
            // the child element collapses and its zero-weight points are
            // skipped, as the reference's iterative root lands there too.
            const double tol = 8.0 * std::numeric_limits<double>::epsilon() *
                               (std::fabs(m.x[b] - m.x[a]) + std::fabs(m.y[b] - m.y[a]) + std::fabs(m.x[b]) + std::fabs(m.y[b]));
            for (int end : {a, b})
                if (std::fabs(ex - m.x[end]) + std::fabs(ey - m.y[end]) <= tol) { ex = m.x[end]; ey = m.y[end]; }
            for (int copy = 0; copy < (spec.cohesive ? 2 : 1); ++copy) {
                const int idx = k + copy * m.n_enr_initial;
                m.x[m.n_reg + idx] = ex;
                m.y[m.n_reg + idx] = ey;
                m.enr_edge[2 * idx] = a;
                m.enr_edge[2 * idx + 1] = b;
                m.enr_inc[idx] = inc;
            }
            ++k;
        }
    }
    m.cut_enr.assign((size_t)m.n_cut * kMaxEnr, -1);
    for (int c = 0; c < m.n_cut; ++c) {
        const int e = m.cut_elem[c];
        const CutTemplate& T = templates()[m.cut_tmpl[c]];
        for (int s = 0; s < T.n_cut_edges; ++s) {
            int a = m.conn[3 * e + kEdgeNodes[T.cut_edge[s]][0]], b = m.conn[3 * e + kEdgeNodes[T.cut_edge[s]][1]];
            if (a > b) std::swap(a, b);
            const EdgeKey key{{a, b}, slot_inc[c * 6 + s]};
            const int k = (int)(std::lower_bound(cut_edges.begin(), cut_edges.end(), key) - cut_edges.begin());
            m.cut_enr[(size_t)c * kMaxEnr + s] = m.n_reg + k;
            if (spec.cohesive) m.cut_enr[(size_t)c * kMaxEnr + s + T.n_cut_edges] = m.n_reg + k + m.n_enr_initial;
        }
    }

    // ---- Dirichlet data (Tests/Main.cpp:444-450) and reference DOF numbering ----
    const int nn = m.n_nodes();
    m.fixed.assign(2 * (size_t)nn, 0);
    m.ubar.assign(2 * (size_t)nn, 0.0);
    const double app = (spec.x1 - spec.x0) * spec.strain;
    for (int j = 0; j <= ny; ++j) {
        const int left = j * (nx + 1), right = nx + j * (nx + 1);
        m.fixed[2 * left] = 1;
        m.ubar[2 * left] = 0.0;
        m.fixed[2 * right] = 1;
        m.ubar[2 * right] = app;
    }
    m.fixed[0] = m.fixed[1] = 1;
    m.ubar[0] = m.ubar[1] = 0.0;
    int n_reg_free = 0;
    for (int i = 0; i < 2 * m.n_reg; ++i) n_reg_free += !m.fixed[i];
    m.n_free = n_reg_free + 2 * m.n_enr;
    m.ref_dof.resize(2 * (size_t)nn);
    {
        int f = 0, p = 0;
        for (int i = 0; i < 2 * m.n_reg; ++i) m.ref_dof[i] = m.fixed[i] ? m.n_free + p++ : f++;
        for (int i = 2 * m.n_reg; i < 2 * nn; ++i) m.ref_dof[i] = f++;
    }

    // ---- 2x2-block sparsity over nodes ----
    // The pattern is the union of every element's node pairs.  On the
    // structured background grid a regular node's row holds its grid
    // neighbours -- the four axis neighbours inside the grid, and the four
    // diagonal ones for even nodes ((i + j) % 2 == 0), the only nodes a cell
    // diagonal passes through -- in index order, then the enrichment nodes of
    // the cut elements it belongs to; an enrichment node's row holds the
    // local nodes of its cut elements.  Only those lists need sorting.
    std::vector<int> cut_L((size_t)m.n_cut * kMaxElemNodes), cut_nl(m.n_cut);
    for (int c = 0; c < m.n_cut; ++c) {
        const int e = m.cut_elem[c];
        const CutTemplate& T = templates()[m.cut_tmpl[c]];
        int* L = &cut_L[(size_t)c * kMaxElemNodes];
        cut_nl[c] = 3 + T.n_enr;
        for (int v = 0; v < 3; ++v) L[v] = m.conn[3 * e + v];
        for (int s = 0; s < T.n_enr; ++s) L[3 + s] = m.cut_enr[(size_t)c * kMaxEnr + s];
    }
    std::vector<int> xptr(nn + 1, 0);
    for (int c = 0; c < m.n_cut; ++c)
        for (int a = 0; a < cut_nl[c]; ++a) {
            const int na = cut_L[(size_t)c * kMaxElemNodes + a];
            xptr[na + 1] += na < m.n_reg ? cut_nl[c] - 3 : cut_nl[c];
        }
    for (int n = 0; n < nn; ++n) xptr[n + 1] += xptr[n];
    std::vector<int> xcol(xptr.back());
    {
        std::vector<int> fill(xptr.begin(), xptr.end() - 1);
        for (int c = 0; c < m.n_cut; ++c) {
            const int* L = &cut_L[(size_t)c * kMaxElemNodes];
            for (int a = 0; a < cut_nl[c]; ++a)
                for (int b = L[a] < m.n_reg ? 3 : 0; b < cut_nl[c]; ++b) xcol[fill[L[a]]++] = L[b];
        }
    }
    std::vector<int> xlen(nn, 0);
    for (int n = 0; n < nn; ++n) {
        int* b = xcol.data() + xptr[n];
        int* e = xcol.data() + xptr[n + 1];
        if (b == e) continue;
        std::sort(b, e);
        xlen[n] = (int)(std::unique(b, e) - b);
    }
    // grid neighbours of node (gi, gj) as bits d = 3 (dy + 1) + (dx + 1)
    auto nbr_mask = [nx, ny](int gi, int gj) {
        const bool even = ((gi + gj) & 1) == 0;
        const bool w = gi > 0, ea = gi < nx, so = gj > 0, no = gj < ny;
        return (so && even && w ? 1u : 0u) | (so ? 2u : 0u) | (so && even && ea ? 4u : 0u) | (w ? 8u : 0u) | 16u |
               (ea ? 32u : 0u) | (no && even && w ? 64u : 0u) | (no ? 128u : 0u) | (no && even && ea ? 256u : 0u);
    };
    m.row_ptr.assign(nn + 1, 0);
    for (int n = 0; n < nn; ++n) {
        const int reg = n < m.n_reg ? __builtin_popcount(nbr_mask(n % (nx + 1), n / (nx + 1))) : 0;
        m.row_ptr[n + 1] = m.row_ptr[n] + reg + xlen[n];
    }
    m.col.resize(m.row_ptr.back());
    m.diag_slot.resize(nn);
    for (int n = 0; n < nn; ++n) {
        int q = m.row_ptr[n];
        if (n < m.n_reg) {
            const int gi = n % (nx + 1), gj = n / (nx + 1);
            const unsigned mask = nbr_mask(gi, gj);
            for (int d = 0; d < 9; ++d)
                if (mask & (1u << d)) m.col[q++] = (gi + d % 3 - 1) + (gj + d / 3 - 1) * (nx + 1);
        }
        std::copy(xcol.data() + xptr[n], xcol.data() + xptr[n] + xlen[n], m.col.begin() + q);
        const int* b = m.col.data() + m.row_ptr[n];
        const int* e = m.col.data() + m.row_ptr[n + 1];
        m.diag_slot[n] = (int)(std::lower_bound(b, e, n) - m.col.data());
    }
    auto slot_of = [&](int r, int c) -> int {
        const int* b = m.col.data() + m.row_ptr[r];
        const int* e = m.col.data() + m.row_ptr[r + 1];
        const int* it = std::lower_bound(b, e, c);
        return (it != e && *it == c) ? (int)(it - m.col.data()) : -1;
    };

    // per node: adjacent uncut elements with the node's local vertex (empty
    // for enrichment nodes, whose rows only the cut-element kernel fills)
    m.ne_ptr.assign(nn + 1, 0);
    for (int e = 0; e < m.n_elem; ++e)
        if (m.elem_cut[e] < 0)
            for (int v = 0; v < 3; ++v) m.ne_ptr[m.conn[3 * e + v] + 1]++;
    for (int n = 0; n < nn; ++n) m.ne_ptr[n + 1] += m.ne_ptr[n];
    m.ne_list.resize(m.ne_ptr.back());
    {
        std::vector<int> fill(m.ne_ptr.begin(), m.ne_ptr.end() - 1);
        for (int e = 0; e < m.n_elem; ++e)
            if (m.elem_cut[e] < 0)
                for (int v = 0; v < 3; ++v) m.ne_list[fill[m.conn[3 * e + v]]++] = (e << 2) | v;
    }

    // per cut element: block slots of every local (a, b) pair
    constexpr int S = kMaxElemNodes;
    m.cut_slot.assign((size_t)m.n_cut * S * S, -1);
    m.cut_coh_qp0.resize(m.n_cut);
    for (int c = 0; c < m.n_cut; ++c) {
        const int e = m.cut_elem[c];
        const CutTemplate& T = templates()[m.cut_tmpl[c]];
        int L[kMaxElemNodes];
        const int nl = 3 + T.n_enr;
        for (int v = 0; v < 3; ++v) L[v] = m.conn[3 * e + v];
        for (int s = 0; s < T.n_enr; ++s) L[3 + s] = m.cut_enr[(size_t)c * kMaxEnr + s];
        for (int a = 0; a < nl; ++a)
            for (int b = 0; b < nl; ++b) m.cut_slot[(size_t)c * S * S + a * S + b] = slot_of(L[a], L[b]);
        m.cut_coh_qp0[c] = m.n_coh_qp;
        m.n_coh_qp += 2 * T.n_coh;
    }
    return std::string();
}

}  // namespace pgb
