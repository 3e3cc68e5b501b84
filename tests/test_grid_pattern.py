"""Host logic behind the structured-grid assembly kernel (`k_assemble_grid`),
checked on CPU: on every structured mesh the host builds, the block row of a
regular node (i, j) holds exactly its grid neighbours (all four axis
neighbours inside the grid, the four diagonal ones only where i + j is even)
and itself, in ascending node order, followed only by enrichment columns.

The kernel relies on this layout to find every block's place in its row from
the node's neighbour mask, with no per-block map (`grid_pattern_ok` checks it
again in C++ when a context is made and falls back to the gather kernel)."""
import numpy as np
import pytest

import pigfem_assignment_b200.problem as pb
from pigfem_assignment_b200.rve import RVE, config0, config2


def neighbour_row(gi, gj, nx, ny):
    even = (gi + gj) % 2 == 0
    out = []
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            i, j = gi + dx, gj + dy
            if not (0 <= i <= nx and 0 <= j <= ny):
                continue
            if dx != 0 and dy != 0 and not even:
                continue
            out.append(i + j * (nx + 1))
    return out


def check_layout(rve):
    e = pb.Mesh(rve).export()
    nx, ny = rve.nx, rve.ny
    rp, col = e["row_ptr"], e["col"]
    n_reg = e["n_regular_nodes"]
    assert n_reg == (nx + 1) * (ny + 1)
    enr_rows = 0
    for gj in range(ny + 1):
        for gi in range(nx + 1):
            node = gi + gj * (nx + 1)
            row = list(col[rp[node]:rp[node + 1]])
            want = neighbour_row(gi, gj, nx, ny)
            assert row[:len(want)] == want, (gi, gj, row, want)
            tail = row[len(want):]
            assert all(c >= n_reg for c in tail), (gi, gj, tail)
            assert tail == sorted(tail)
            enr_rows += bool(tail)
    return enr_rows


@pytest.mark.parametrize("rve", [
    config0(),
    RVE(nx=70, ny=37, inclusions=[(0.5, 0.5, 0.25, 1)], strain=0.01),
    RVE(nx=40, ny=45, inclusions=[(0.3, 0.3, 0.12, 1), (0.72, 0.66, 0.17, 1), (0.1, 0.85, 0.08, 1)], strain=0.01),
    RVE(nx=31, ny=2, inclusions=[(0.5, 0.5, 0.3, 1)], strain=0.01),
    config2(nx=48, n_inc=6),
], ids=["config0", "70x37", "40x45-three", "31x2", "cohesive-48"])
def test_regular_rows_follow_the_grid_layout(rve):
    # cut elements put enrichment columns into some regular rows; the test needs meshes that have them
    assert check_layout(rve) > 0
