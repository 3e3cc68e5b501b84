// Writers of a context's state: the reference's legacy ASCII VTK file
// (Writer_ASCII_VTK over Writer_VTK: Writer_ASCII_VTK.cpp:58-387,
// Writer_VTK.cpp:164-336, 639-911) and its cohesive openings CSV
// (WriterCohesiveOpenings.cpp:39-197).  Off the timed path: the device forms
// the displacement and the strain and stress of every quadrature point
// (stress_strain), the host formats the text.
//
// The files hold what the reference's do, value for value and in the same
// order and number format (floats through an ostream at its default
// precision; the CSV at precision 16):
//   POINTS        regular nodes, then enrichment nodes (cohesive mirror nodes
//                 after the originals), as floats with z = 0
//   CELLS         every uncut element, and in place of a cut element its
//                 integration children in template order (VTK triangle 5,
//                 quad 9, polygon 7)
//   POINT_DATA    displacement and external_force (3 floats per node); at an
//                 enrichment node, the parent edge's interpolation plus the
//                 node's own value (Problem::interpolate_nodal_enrichment,
//                 Problem.cpp:656-685, with Mesh::compute_enrich_node_
//                 interpolation's ratio, Mesh.cpp:3663-3690)
//   CELL_DATA     the reference's material number, partitions (0), the
//                 arithmetic means of strain and stress over the cell's
//                 quadrature points (accumulated in float as the reference
//                 does) and the von Mises stress of the mean stress
// The external force is the solver's F_ext: zero on free DOFs (these RVEs
// carry no applied loads) and the reaction on prescribed ones
// (SolverLinear.cpp:131-143, SolverNonlinear.cpp:339-341).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "pg_internal.cuh"

namespace pgb {

namespace {

int child_type_of(int nc) { return nc == 3 ? kChildTri3 : nc == 4 ? kChildQuad4 : nc == 5 ? kChildPoly5 : kChildPoly6; }
int vtk_cell_type(int nc) { return nc == 3 ? 5 : nc == 4 ? 9 : 7; }

// The reference's material numbers: Mesh::add_inclusion adds each inclusion's
// material the first time an inclusion uses it (Mesh.cpp:2590-2622), the
// matrix material is added after the mesh is generated, the cohesive law last.
std::vector<int> reference_material_numbers(const RveSpec& s) {
    std::vector<int> id(s.materials.size() + 1, -1);
    int next = 0;
    for (const Inclusion& inc : s.inclusions)
        if (inc.mat >= 0 && inc.mat < (int)s.materials.size() && id[inc.mat] < 0 && inc.mat != s.matrix_mat)
            id[inc.mat] = next++;
    if (s.matrix_mat >= 0 && s.matrix_mat < (int)s.materials.size()) id[s.matrix_mat] = next++;
    for (int& v : id)
        if (v < 0) v = next;  // unused by the mesh
    return id;
}

// Mesh::compute_enrich_node_interpolation: the enrichment node's position
// along its parent edge, averaged over the coordinates in which the edge
// moves (a coordinate counts when |diff / x1| or |diff / x2| exceeds 1e-10)
double edge_ratio(double x1, double y1, double x2, double y2, double ex, double ey) {
    const double c1[2] = {x1, y1}, c2[2] = {x2, y2}, e[2] = {ex, ey};
    double ratio = 0.0;
    int count = 0;
    for (int d = 0; d < 2; ++d) {
        const double diff = c2[d] - c1[d];
        double k1 = diff / c1[d];
        if (k1 < 0.0) k1 = -k1;
        double k2 = diff / c2[d];
        if (k2 < 0.0) k2 = -k2;
        if (k1 > 1e-10 || k2 > 1e-10) {
            ratio += (e[d] - c1[d]) / diff;
            ++count;
        }
    }
    return ratio / count;
}

// Utilities::von_mises for three float components, with its float and
// double steps (Utilities.cpp:713-723)
float von_mises3(const float s[3]) {
    const float a = s[0] * s[0] - s[0] * s[1] + s[1] * s[1];
    return (float)std::sqrt((double)a + 3.0 * (double)s[2] * (double)s[2]);
}

// Per node (3 floats): the nodal field v (2 per node, library DOF order) with
// the enrichment nodes' parent-edge interpolation added
std::vector<float> nodal_plot_field(const HostMesh& m, const std::vector<double>& v) {
    const int nn = m.n_nodes();
    std::vector<float> out(3 * (size_t)nn, 0.0f);
    for (int n = 0; n < m.n_reg; ++n)
        for (int d = 0; d < 2; ++d) out[3 * (size_t)n + d] = (float)v[2 * (size_t)n + d];
    for (int k = 0; k < m.n_enr; ++k) {
        const int n = m.n_reg + k, a = m.enr_edge[2 * k], b = m.enr_edge[2 * k + 1];
        const double t = edge_ratio(m.x[a], m.y[a], m.x[b], m.y[b], m.x[n], m.y[n]);
        for (int d = 0; d < 2; ++d)
            out[3 * (size_t)n + d] = (float)(v[2 * (size_t)a + d] * (1.0 - t) + v[2 * (size_t)b + d] * t +
                                             v[2 * (size_t)n + d]);
    }
    return out;
}

int download(std::vector<double>& h, const double* d, size_t n, cudaStream_t s) {
    h.resize(n);
    PG_CUDA(cudaMemcpyAsync(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    PG_CUDA(cudaStreamSynchronize(s));
    return PG_OK;
}

}  // namespace

int write_vtk(Ctx& c, const std::string& path, double t) {
    const HostMesh& m = c.hm;
    cudaStream_t s = c.stream;
    // the reactions: a linear mesh's solve leaves no internal force behind,
    // so form F_int = K U here; a cohesive mesh keeps the last residual's
    if (!m.spec.cohesive) {
        PG_CUDA(cudaMemsetAsync(c.F, 0, (size_t)c.n_dof * sizeof(double), s));
        int rc = launch_assemble(c, c.U, 0.0, true, false, s);
        if (rc != PG_OK) return rc;
    }
    int rc = stress_strain(c, c.U, s, nullptr);
    if (rc != PG_OK) return rc;
    std::vector<double> U, F, pts;
    if ((rc = download(U, c.U, (size_t)c.n_dof, s)) || (rc = download(F, c.F, (size_t)c.n_dof, s)) ||
        (rc = download(pts, c.qp_out, 7 * (size_t)c.n_qp_total, s)))
        return rc;
    std::vector<int> qp_off(m.n_elem + 1);
    PG_CUDA(cudaMemcpy(qp_off.data(), c.qp_off, qp_off.size() * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < c.n_dof; ++i)
        if (!m.fixed[i]) F[i] = 0.0;

    std::ofstream out(path, std::ofstream::out);
    if (!out.good()) {
        set_error("pg_write_vtk: cannot open " + path);
        return PG_ERR_ARG;
    }
    const std::vector<int> mat_no = reference_material_numbers(m.spec);
    // Writer_ASCII_VTK::write_header
    out << "# vtk DataFile Version 3.0\n";
    out << "IGFEM 2D simulation: t=" << t << "\n";
    out << "ASCII\n\n";
    out << "DATASET UNSTRUCTURED_GRID\n";
    // write_nodes
    const int nn = m.n_nodes();
    out << "POINTS " << nn << " float\n";
    for (int n = 0; n < nn; ++n) out << (float)m.x[n] << " " << (float)m.y[n] << " " << 0.0f << "\n";
    // Writer_VTK::store_elements: cells, their types and materials, and the
    // quadrature points each cell averages over
    std::vector<int> cell_ptr(1, 0), cell_nodes, cell_type, cell_mat, cell_qp0, cell_nq;
    for (int e = 0; e < m.n_elem; ++e) {
        const int ci = m.elem_cut[e];
        if (ci < 0) {
            for (int v = 0; v < 3; ++v) cell_nodes.push_back(m.conn[3 * (size_t)e + v]);
            cell_type.push_back(5);
            cell_mat.push_back(mat_no[m.elem_mat[e]]);
            cell_qp0.push_back(qp_off[e]);
            cell_nq.push_back(qp_off[e + 1] - qp_off[e]);
            cell_ptr.push_back((int)cell_nodes.size());
            continue;
        }
        const CutTemplate& T = cut_template(m.cut_tmpl[ci]);
        int q0 = qp_off[e];
        for (int ch = 0; ch < T.n_child; ++ch) {
            const int nc = T.child_n[ch];
            for (int k = 0; k < nc; ++k) {
                const int ln = T.child_nodes[ch][k];
                cell_nodes.push_back(ln < 3 ? m.conn[3 * (size_t)e + ln] : m.cut_enr[(size_t)kMaxEnr * ci + ln - 3]);
            }
            const int nq = child_quadrature(child_type_of(nc)).nq;
            cell_type.push_back(vtk_cell_type(nc));
            const int cm = m.cut_child_mat[(size_t)kMaxChildren * ci + ch];
            cell_mat.push_back(mat_no[cm]);
            cell_qp0.push_back(q0);
            cell_nq.push_back(nq);
            q0 += nq;
            cell_ptr.push_back((int)cell_nodes.size());
        }
    }
    const size_t n_cells = cell_type.size();
    // write_elements
    out << "\nCELLS " << n_cells << " " << (n_cells + cell_nodes.size()) << "\n";
    for (size_t k = 0; k < n_cells; ++k) {
        out << (cell_ptr[k + 1] - cell_ptr[k]) << " ";
        for (int i = cell_ptr[k]; i < cell_ptr[k + 1]; ++i) out << cell_nodes[i] << (i == cell_ptr[k + 1] - 1 ? "\n" : " ");
    }
    out << "\nCELL_TYPES " << n_cells << "\n";
    for (size_t k = 0; k < n_cells; ++k) out << cell_type[k] << "\n";
    // write_nodal_data
    const std::vector<float> sol = nodal_plot_field(m, U), rhs = nodal_plot_field(m, F);
    out << "\nPOINT_DATA " << nn << "\n";
    out << "VECTORS displacement float " << "\n";
    for (int n = 0; n < nn; ++n) out << sol[3 * (size_t)n] << " " << sol[3 * (size_t)n + 1] << " " << sol[3 * (size_t)n + 2] << "\n";
    out << "VECTORS external_force float " << "\n";
    for (int n = 0; n < nn; ++n) out << rhs[3 * (size_t)n] << " " << rhs[3 * (size_t)n + 1] << " " << rhs[3 * (size_t)n + 2] << "\n";
    // gather_element_data: float means over the cell's points
    std::vector<float> avg(6 * n_cells, 0.0f);
    for (size_t k = 0; k < n_cells; ++k)
        for (int v = 0; v < 6; ++v) {
            float a = 0.0f;
            for (int q = 0; q < cell_nq[k]; ++q) a += pts[7 * ((size_t)cell_qp0[k] + q) + v];
            avg[6 * k + v] = a / cell_nq[k];
        }
    // write_element_data
    out << "\nCELL_DATA " << n_cells << "\n";
    out << "SCALARS materials int\n";
    out << "LOOKUP_TABLE default\n";
    for (size_t k = 0; k < n_cells; ++k) out << cell_mat[k] << "\n";
    out << "\nSCALARS partitions int\n";
    out << "LOOKUP_TABLE default\n";
    for (size_t k = 0; k < n_cells; ++k) out << 0 << "\n";
    static const char* kVoigt[3] = {"11", "22", "12"};
    for (int part = 0; part < 2; ++part)
        for (int v = 0; v < 3; ++v) {
            out << "\nSCALARS " << (part == 0 ? "e" : "s") << kVoigt[v] << " float\n";
            out << "LOOKUP_TABLE default\n";
            for (size_t k = 0; k < n_cells; ++k) out << avg[6 * k + 3 * part + v] << "\n";
        }
    out << "\nSCALARS von_mises float\n";
    out << "LOOKUP_TABLE default\n";
    for (size_t k = 0; k < n_cells; ++k) out << von_mises3(&avg[6 * k + 3]) << "\n";
    out.close();
    if (!out) {
        set_error("pg_write_vtk: write failed: " + path);
        return PG_ERR_ARG;
    }
    return PG_OK;
}

int write_cohesive_openings(Ctx& c, const std::string& path) {
    const HostMesh& m = c.hm;
    if (!m.spec.cohesive) {
        set_error("pg_write_cohesive_openings: the mesh has no cohesive interface");
        return PG_ERR_ARG;
    }
    // the law's critical openings (normal, tangential): the Ortiz-Pandolfi
    // law's delta_c for both (WriterCohesiveOpenings.cpp:100-104); for the
    // bilinear law its final opening 2 G_c / sigma_c
    const CohesiveLaw& law = m.spec.coh;
    const double dc = law.law == 0 ? law.p[1] : 2.0 * law.p[1] / law.p[0];
    std::vector<double> U;
    int rc = download(U, c.U, (size_t)c.n_dof, c.stream);
    if (rc != PG_OK) return rc;
    std::vector<std::tuple<int, double, double, double>> rows;
    for (int e = 0; e < m.n_elem; ++e) {
        const int ci = m.elem_cut[e];
        if (ci < 0) continue;
        const CutTemplate& T = cut_template(m.cut_tmpl[ci]);
        for (int ce = 0; ce < T.n_coh; ++ce) {
            int n[4];
            for (int k = 0; k < 4; ++k) {
                const int ln = T.coh_nodes[ce][k];
                n[k] = ln < 3 ? m.conn[3 * (size_t)e + ln] : m.cut_enr[(size_t)kMaxEnr * ci + ln - 3];
            }
            const int inc = m.enr_inc[n[0] - m.n_reg];
            const Inclusion& I = m.spec.inclusions[inc];
            // midpoint of the lower surface, its angle about the centre
            double mx = 0.0, my = 0.0;
            mx += 0.5 * m.x[n[0]];
            mx += 0.5 * m.x[n[1]];
            my += 0.5 * m.y[n[0]];
            my += 0.5 * m.y[n[1]];
            const double theta = std::atan2(my - I.cy, mx - I.cx);
            // opening at the midpoint (ProblemUtilities::cohesiveDeltaFast,
            // Utilities.cpp:465-477) in the element's frame
            double dg[2] = {0.0, 0.0};
            for (int d = 0; d < 2; ++d) {
                dg[d] += 0.5 * (U[2 * (size_t)n[2] + d] - U[2 * (size_t)n[0] + d]);
                dg[d] += 0.5 * (U[2 * (size_t)n[3] + d] - U[2 * (size_t)n[1] + d]);
            }
            const double jx = 0.5 * (m.x[n[1]] - m.x[n[0]]), jy = 0.5 * (m.y[n[1]] - m.y[n[0]]);
            const double mag = std::sqrt(jx * jx + jy * jy);
            const double tn = (jx / mag) * dg[0] + (jy / mag) * dg[1];
            const double nr = (-jy / mag) * dg[0] + (jx / mag) * dg[1];
            rows.emplace_back(inc, theta, tn / dc, nr / dc);
        }
    }
    std::sort(rows.begin(), rows.end());
    std::ofstream out(path, std::ofstream::out);
    if (!out.good()) {
        set_error("pg_write_cohesive_openings: cannot open " + path);
        return PG_ERR_ARG;
    }
    out.precision(16);
    for (const auto& r : rows)
        out << std::get<0>(r) << "," << std::get<1>(r) << "," << std::get<2>(r) << "," << std::get<3>(r) << "\n";
    out.close();
    if (!out) {
        set_error("pg_write_cohesive_openings: write failed: " + path);
        return PG_ERR_ARG;
    }
    return PG_OK;
}

}  // namespace pgb
