// Host-side IGFEM preprocessing for the B200 assembly/solve path.
//
// Restates, for structured TRI3 meshes cut by circular inclusions, what the
// reference does once per mesh before any assembly:
//   Mesh::generate_mesh (TRI3)          PIGFEM4.6.1/src/Mesh.cpp:191-405
//   Mesh::analyze_nodes / detect_node   Mesh.cpp:2676-2714, 2838-2918
//   Tri3::detection (cut templates)     tri3.cpp:287-541
//   Mesh::analyze_elements              Mesh.cpp:2922-3027
//   Mesh::add_enrichments (serial)      Mesh.cpp:3038-3202, 3600-3660
//   Inclusion::find_intersection        Inclusion.cpp:32-128, InclusionCircle.cpp:248-287
//   DofObject::distribute_dofs          DofObject.cpp:241-386
//   Solver::preallocate_matrix sparsity Solver.cpp:365-441, 723-829
// and lays the result out flat for the device: structure-of-arrays node
// coordinates, a 2x2-block CSR pattern over all nodes, per-node lists of the
// uncut elements around it, and compact descriptors of the cut elements.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pgb {

constexpr int kMaxEnr = 12;          // enrichment slots of one cut element (3 cut edges x 2 surfaces x 2)
constexpr int kMaxElemNodes = 3 + kMaxEnr;
constexpr int kMaxChildren = 4;
constexpr int kMaxChildNodes = 6;
constexpr int kMaxCoh = 3;

// Child (integration sub-element) types and the shape of the tables the
// device uses to integrate them.
enum ChildType : int { kChildTri3 = 0, kChildQuad4 = 1, kChildPoly5 = 2, kChildPoly6 = 3, kNumChildTypes = 4 };

// A cut-element template: the restated content of one branch of
// Tri3::detection.  Local node numbering: 0..2 parent nodes, 3.. enrichment
// slots (mirror slots follow the lower-surface slots for cohesive meshes).
struct CutTemplate {
    int n_cut_edges;                   // |_cutEdge|
    int n_enr;                         // enrichment slots = n_cut_edges (x2 if cohesive)
    int cut_edge[6];                   // parent edge of each cut-edge slot (edge e joins nodes e, (e+1)%3)
    int enr_inc_node[6];               // slot's inclusion = detection value of this parent node (-1: max of the element's values)
    int n_child;
    int child_n[kMaxChildren];
    int child_nodes[kMaxChildren][kMaxChildNodes];
    int child_mat_node[kMaxChildren];  // child material = material of this parent node's region; -1 = element (matrix) material
    int n_coh;
    int coh_nodes[kMaxCoh][4];
};

struct Inclusion {
    double cx, cy, r;
    int mat;
};

struct Material {
    double E, nu;
};

// Cohesive law parameters.  law 0: Ortiz-Pandolfi exponential with linear
// unloading and viscous regularisation (the reference's active law,
// Material_OPCohesive.cpp:38-253): p = {sigma_c, delta_c, beta, viscosity}.
// law 1: bilinear penalty law: p = {sigma_c, G_c, K_p, beta, eta} with the
// viscous traction eta (delta_eff - delta_max) / dt while loading.
struct CohesiveLaw {
    int law = 0;
    double p[5] = {0, 0, 0, 0, 0};
};

struct RveSpec {
    int nx = 64, ny = 64;
    double x0 = 0, x1 = 1, y0 = 0, y1 = 1;
    std::vector<Inclusion> inclusions;
    std::vector<Material> materials;   // materials[matrix_mat] is the matrix
    int matrix_mat = 0;
    bool cohesive = false;
    CohesiveLaw coh;
    double strain = 0.01;              // right edge u_x = (x1-x0)*strain (scaled by the load factor)
    bool plane_strain = true;
};

struct HostMesh {
    RveSpec spec;
    // nodes: regular nodes 0..n_reg-1, then enrichment nodes
    int n_reg = 0, n_enr = 0, n_enr_initial = 0;
    std::vector<double> x, y;
    std::vector<int> node_detect;          // per regular node: inclusion id or -1
    int n_moved = 0;                       // nodes moved off an inclusion surface
    // elements
    int n_elem = 0;
    std::vector<int> conn;                 // 3 per element
    std::vector<int> elem_mat;             // material of an uncut element; matrix material for cut ones
    std::vector<int> elem_cut;             // -1 or index into the cut arrays
    // cut elements
    int n_cut = 0;
    std::vector<int> cut_elem, cut_tmpl;
    std::vector<int> cut_enr;              // kMaxEnr per cut element: global node index of each slot, -1 unused
    std::vector<int> cut_child_mat;        // kMaxChildren per cut element
    std::vector<int> cut_coh_mat;          // kMaxCoh per cut element (index into the cohesive law list; 0)
    // enrichment nodes
    std::vector<int> enr_edge;             // 2 per enrichment node (sorted regular node ids)
    std::vector<int> enr_inc;
    // Dirichlet data (per DOF = 2*node + d)
    std::vector<uint8_t> fixed;
    std::vector<double> ubar;              // full prescribed value (load factor 1)
    // reference DOF numbering (free regular DOFs, enrichment DOFs, then prescribed)
    std::vector<int> ref_dof;
    int n_free = 0;
    // 2x2-block CSR pattern over all nodes
    std::vector<int> row_ptr, col, diag_slot;
    // per node: adjacent uncut elements, packed (elem << 2) | local vertex
    std::vector<int> ne_ptr, ne_list;
    // per cut element: block slots for every (local a, local b), (3+kMaxEnr)^2 entries, -1 unused
    std::vector<int> cut_slot;
    // cohesive quadrature points (2 per cohesive sub-element)
    int n_coh_qp = 0;
    std::vector<int> cut_coh_qp0;          // first cohesive qp index of each cut element
    // the structured background grids the mesh is made of: one for a mesh
    // built here, one per RVE in a merged batch (its regular nodes and
    // elements from the offsets on, its enrichment nodes after them)
    struct GridBlock {
        int nx, ny, node_off, elem_off, n_reg;
    };
    std::vector<GridBlock> grids;

    int n_nodes() const { return n_reg + n_enr; }
    int n_dof() const { return 2 * n_nodes(); }
    int n_blocks() const { return row_ptr.empty() ? 0 : row_ptr.back(); }
};

const CutTemplate& cut_template(int id);
int n_cut_templates();

// Builds the enriched mesh, DOF maps and sparsity.  Returns an empty string
// on success, otherwise a description of the failure (the reference would
// call err_message and exit; this never exits).
std::string build_mesh(const RveSpec& spec, HostMesh& out);

// Reference quadrature tables per child type (restated from Tri3::q_point
// order 3, Quad4::q_point order 3, Polygon::q_point with the reference's
// order mismatch: n_q_points(order 3) points drawn from the order-5 rule).
struct ChildQuadrature {
    int nq;
    int nn;
    std::vector<double> w;        // nq
    std::vector<double> N;        // nq * nn
    std::vector<double> dN;       // nq * nn * 2 (d/dxi, d/deta)
};
const ChildQuadrature& child_quadrature(int type);

}  // namespace pgb
