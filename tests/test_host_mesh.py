"""The product's host IGFEM preprocessing against the reference's own
enriched mesh (golden fixtures), and its K through the pinned oracle."""
import numpy as np
import pytest

import oracle
import pigfem_assignment_b200.problem as pb
from helpers import golden, permute_to_ref, ref_full_K, rel_fro, rve_from_golden
from pigfem_assignment_b200.rve import SplitMix64, config0, config1, rsa_circles

CASES = [("linear_8x8.npz", False), ("linear_cfg0.npz", False), ("linear_3inc.npz", False),
         ("cohesive_16x16.npz", True)]


@pytest.mark.parametrize("name,coh", CASES)
def test_enriched_mesh_matches_reference(name, coh):
    g = golden(name)
    rve = rve_from_golden(g, cohesive=coh)
    m = pb.Mesh(rve)
    e = m.export()
    nreg = e["n_regular_nodes"]
    ref_xy = g["mesh.node_xy"].reshape(-1, 2)
    ref_exy = g["mesh.enr_xy"].reshape(-1, 2)
    assert nreg == ref_xy.shape[0]
    assert m.info["n_enrichment_nodes"] == ref_exy.shape[0]
    # regular nodes (including the ones moved off an interface) are identical
    np.testing.assert_array_equal(e["xy"][:nreg], ref_xy)
    # enrichment nodes: the reference's iterative root vs a closed-form root
    assert np.abs(e["xy"][nreg:] - ref_exy).max() <= 1e-12
    np.testing.assert_array_equal((e["elem_cut"] >= 0).astype(np.int32), g["mesh.is_cut"])
    ptr, ce = g["mesh.cut_enr_ptr"], g["mesh.cut_enr"]
    for c, el in enumerate(e["cut_elem"]):
        ref = ce[ptr[el]:ptr[el + 1]]
        np.testing.assert_array_equal(e["cut_enr"][c][: ref.size] - nreg, ref)
    np.testing.assert_array_equal(e["ref_dof"], np.concatenate([g["dof.node"], g["dof.enr"]]))
    assert e["n_free"] == int(g["dof.n_free"][0])


@pytest.mark.parametrize("name,coh", CASES)
def test_templates_and_materials_match_reference(name, coh):
    g = golden(name)
    rve = rve_from_golden(g, cohesive=coh)
    m = pb.Mesh(rve)
    e = m.export()
    T = pb.template_table()
    cp, cnp, cn, cm = g["mesh.child_ptr"], g["mesh.child_nodes_ptr"], g["mesh.child_nodes"], g["mesh.child_mat"]
    hp, hn = g["mesh.coh_ptr"], g["mesh.coh_nodes"]
    refE = g["mesh.mat_E"]
    myE = np.array([mm[0] for mm in rve.materials])
    for c, el in enumerate(e["cut_elem"]):
        t = T[e["cut_tmpl"][c]]
        kids = [list(t[24 + 6 * k: 24 + 6 * k + t[16 + k]]) for k in range(t[2])]
        ref_kids = [list(cn[cnp[i]:cnp[i + 1]]) for i in range(cp[el], cp[el + 1])]
        assert kids == ref_kids
        mats = [myE[e["cut_child_mat"][c][k]] for k in range(t[2])]
        assert mats == [refE[cm[i]] for i in range(cp[el], cp[el + 1])]
        cohs = [list(t[48 + 4 * k: 48 + 4 * k + 4]) for k in range(t[3])]
        assert cohs == [list(hn[4 * i: 4 * i + 4]) for i in range(hp[el], hp[el + 1])]
    uncut = e["elem_cut"] < 0
    np.testing.assert_array_equal(myE[e["elem_mat"][uncut]], refE[g["mesh.elem_mat"][uncut]])


@pytest.mark.parametrize("name", ["linear_8x8.npz", "linear_cfg0.npz", "linear_3inc.npz"])
def test_product_mesh_K_through_oracle_matches_reference(name):
    g = golden(name)
    rve = rve_from_golden(g)
    m = pb.Mesh(rve)
    om = oracle.from_product(m.export(), pb.template_table(), rve)
    K, _, _ = om.assemble()
    assert rel_fro(permute_to_ref(K, om.ref_dof), ref_full_K(g)) <= 1e-12


def test_config0_counts():
    m = pb.Mesh(config0())
    i = m.info
    assert i["n_elements"] == 8192 and i["n_regular_nodes"] == 4225
    assert i["n_free_dof"] == 8751


def test_rsa_reproducible_and_valid():
    a = rsa_circles(11, 30, 0.02, 0.04, 0.005)
    b = rsa_circles(11, 30, 0.02, 0.04, 0.005)
    assert a == b
    for i, (x, y, r) in enumerate(a):
        assert 0.02 <= r <= 0.04 and r + 0.005 <= x <= 1 - r - 0.005 and r + 0.005 <= y <= 1 - r - 0.005
        for (x2, y2, r2) in a[i + 1:]:
            assert np.hypot(x - x2, y - y2) >= r + r2 + 0.005
    s = SplitMix64(0)
    assert s.next_u64() == 0xE220A8397B1DCDAF  # published first output of splitmix64(0)


def test_config1_mesh_builds():
    m = pb.Mesh(config1())
    i = m.info
    assert i["n_elements"] == 524288
    assert i["n_cut_elements"] > 1000 and i["n_enrichment_nodes"] > 1000


def test_mesh_errors_are_status_codes():
    from pigfem_assignment_b200._lib import PgError
    from pigfem_assignment_b200.rve import RVE
    with pytest.raises(PgError):
        pb.Mesh(RVE(nx=0, ny=4))
    with pytest.raises(PgError):
        pb.Mesh(RVE(nx=4, ny=4, inclusions=[(0.5, 0.5, -1.0, 1)]))


@pytest.mark.parametrize("case", ["bonded", "cohesive", "many"])
def test_block_pattern_is_the_union_of_element_node_pairs(case):
    """The host builder writes a regular node's row from its grid neighbours
    and the cut elements' node lists; the pattern must be exactly the sorted
    union of every element's node pairs (uncut triangles: their 3 nodes; cut
    elements: their parents and enrichment nodes)."""
    from pigfem_assignment_b200.rve import RVE
    if case == "bonded":
        rve = RVE(nx=24, ny=20, inclusions=[(0.5, 0.5, 0.25, 1), (0.1, 0.1, 0.05, 1)], strain=0.01)
    elif case == "cohesive":
        rve = RVE(nx=32, ny=32, inclusions=[(0.3, 0.5, 0.2, 1), (0.72, 0.5, 0.2, 1)], cohesive=True, coh_law=1,
                  coh_params=(30.0, 0.01, 1.0e6, 1.0, 200.0), strain=0.01)
    else:
        circ = rsa_circles(7, 30, 0.03, 0.08, 0.01)
        rve = RVE(nx=64, ny=64, inclusions=[(x, y, r, 1) for x, y, r in circ], strain=0.01)
    m = pb.Mesh(rve)
    e = m.export()
    nn = m.info["n_nodes"]
    rows = [set([n]) for n in range(nn)]
    for t, el in enumerate(e["conn"]):
        if e["elem_cut"][t] >= 0:
            continue
        for a in el:
            rows[a].update(int(b) for b in el)
    for c in range(len(e["cut_elem"])):
        nodes = [int(v) for v in e["conn"][e["cut_elem"][c]]] + [int(v) for v in e["cut_enr"][c] if v >= 0]
        for a in nodes:
            rows[a].update(nodes)
    row_ptr, col = e["row_ptr"], e["col"]
    assert row_ptr[-1] == sum(len(r) for r in rows)
    for n in range(nn):
        assert list(col[row_ptr[n]:row_ptr[n + 1]]) == sorted(rows[n]), n
