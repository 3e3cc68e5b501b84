"""Shared helpers of the test-suite: golden fixtures, format conversions."""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def ref_full_K(rec: dict):
    blocks = []
    for n in ("K.ff", "K.fp", "K.pf", "K.pp"):
        m, k = rec[n + ".shape"]
        blocks.append(sp.csr_matrix((rec[n + ".val"], rec[n + ".col"], rec[n + ".rowptr"]), shape=(m, k)))
    return sp.bmat([[blocks[0], blocks[1]], [blocks[2], blocks[3]]]).tocsr()


def permute_to_ref(K, ref_dof):
    n = K.shape[0]
    P = sp.csr_matrix((np.ones(n), (np.asarray(ref_dof), np.arange(n))), shape=(n, n))
    return (P @ K @ P.T).tocsr()


def rel_fro(A, B) -> float:
    return sp.linalg.norm(A - B) / sp.linalg.norm(B)


def bsr_to_csr(row_ptr, col, vals):
    """2x2-block CSR over nodes (values row-major per block) -> DOF-level CSR."""
    row_ptr = np.asarray(row_ptr)
    col = np.asarray(col)
    n = row_ptr.size - 1
    blk_row = np.repeat(np.arange(n), np.diff(row_ptr))
    v = np.asarray(vals).reshape(-1, 4)
    rows = np.concatenate([2 * blk_row, 2 * blk_row, 2 * blk_row + 1, 2 * blk_row + 1])
    cols = np.concatenate([2 * col, 2 * col + 1, 2 * col, 2 * col + 1])
    data = np.concatenate([v[:, 0], v[:, 1], v[:, 2], v[:, 3]])
    return sp.csr_matrix((data, (rows, cols)), shape=(2 * n, 2 * n))


def rve_from_golden(g: dict, cohesive: bool = False):
    from pigfem_assignment_b200.rve import RVE
    incs = g["cfg.inc"]
    mats = [(3000.0, 0.35)]
    inc_list = []
    for (cx, cy, r, E, nu) in incs:
        key = (float(E), float(nu))
        if key not in mats:
            mats.append(key)
        inc_list.append((float(cx), float(cy), float(r), mats.index(key)))
    nx = int(g["cfg.nx"][0])
    rve = RVE(nx=nx, ny=nx, inclusions=inc_list, materials=mats, strain=0.01)
    if cohesive:
        rve.cohesive = True
        rve.coh_law = 0
        rve.coh_params = tuple(float(v) for v in g["cfg.coh"])
    return rve


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
