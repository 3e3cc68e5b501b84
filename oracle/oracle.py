"""CPU oracle for the B200 IGFEM path -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
import this module; the product never does.

Wraps the C restatement oracle/igfem_oracle.c (built into
oracle/_build/liborc.so by build()) and provides:
  * adapters from the reference's own dump (oracle/refio.py) and from the
    product's mesh export to the oracle's explicit mesh description;
  * assembly of K (DOF-level CSR, node-major DOFs 2*node+d) and f_int;
  * the reference's linear solve with a direct sparse factorisation
    (scipy SuperLU standing in for MUMPS Cholesky, src/Solver.cpp:56-142);
  * permutation into the reference's free-first DOF order and its
    K_ff/K_fp/K_pf/K_pp blocks (src/Assembler.cpp:811-831).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "igfem_oracle.c")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liborc.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class _OrcMesh(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int), ("xy", _dp), ("n_elem", C.c_int), ("conn", _ip), ("elem_mat", _ip), ("is_cut", _ip),
        ("enr_ptr", _ip), ("enr", _ip), ("child_ptr", _ip), ("child_nodes_ptr", _ip), ("child_nodes", _ip),
        ("child_mat", _ip), ("coh_ptr", _ip), ("coh_nodes", _ip), ("n_mat", C.c_int), ("mat_E", _dp),
        ("mat_nu", _dp), ("plane_strain", C.c_int), ("coh_law", C.c_int), ("coh_p", C.c_double * 5),
    ]


def build(force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        tmp = LIB + ".tmp"
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", SRC, "-o", tmp, "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_pattern.argtypes = [C.POINTER(_OrcMesh), _ip, _ip]
        _lib.orc_pattern.restype = C.c_int
        _lib.orc_assemble.argtypes = [C.POINTER(_OrcMesh), _ip, _ip, _dp, _dp, C.c_double, _dp, _dp, _dp, C.c_int,
                                      C.c_int]
        _lib.orc_assemble.restype = C.c_int
        _lib.orc_tri3_K.argtypes = [_dp, C.c_double, C.c_double, C.c_int, _dp]
        _lib.orc_tri3_K.restype = None
        _lib.orc_cohesive_law.argtypes = [C.c_int, _dp, C.c_double, C.c_double, _dp, _dp, _dp, _dp]
        _lib.orc_cohesive_law.restype = None
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class OracleMesh:
    """Explicit enriched mesh the C oracle integrates."""

    def __init__(self, xy, conn, elem_mat, is_cut, enr_lists, child_lists, child_mats, coh_lists, mat_E, mat_nu,
                 plane_strain=True, coh_law=0, coh_p=(0, 0, 0, 0), ref_dof=None, n_free=None):
        self.xy = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1)
        self.n_nodes = self.xy.size // 2
        self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
        self.n_elem = self.conn.size // 3
        self.elem_mat = np.ascontiguousarray(elem_mat, dtype=np.int32)
        self.is_cut = np.ascontiguousarray(is_cut, dtype=np.int32)
        ne = self.n_elem
        enr_ptr = np.zeros(ne + 1, np.int32)
        child_ptr = np.zeros(ne + 1, np.int32)
        coh_ptr = np.zeros(ne + 1, np.int32)
        enr, cnp, cn, cm, hn = [], [0], [], [], []
        for e in range(ne):
            el = enr_lists.get(e, ())
            enr.extend(el)
            enr_ptr[e + 1] = len(enr)
            for c, mat in zip(child_lists.get(e, ()), child_mats.get(e, ())):
                cn.extend(c)
                cnp.append(len(cn))
                cm.append(mat)
            child_ptr[e + 1] = len(cm)
            for h in coh_lists.get(e, ()):
                hn.extend(h)
            coh_ptr[e + 1] = len(hn) // 4
        self.enr_ptr, self.child_ptr, self.coh_ptr = enr_ptr, child_ptr, coh_ptr
        self.enr = np.asarray(enr + [0], np.int32)
        self.child_nodes_ptr = np.asarray(cnp, np.int32)
        self.child_nodes = np.asarray(cn + [0], np.int32)
        self.child_mat = np.asarray(cm + [0], np.int32)
        self.coh_nodes = np.asarray(hn + [0, 0, 0, 0], np.int32)
        self.mat_E = np.ascontiguousarray(mat_E, dtype=np.float64)
        self.mat_nu = np.ascontiguousarray(mat_nu, dtype=np.float64)
        self.plane_strain = int(plane_strain)
        self.coh_law = int(coh_law)
        self.coh_p = tuple(float(v) for v in coh_p) + (0.0,) * (5 - len(coh_p))
        self.n_coh_qp = 2 * (len(hn) // 4)
        self.ref_dof = None if ref_dof is None else np.asarray(ref_dof, np.int64)
        self.n_free = n_free
        self._pattern = None

    def _struct(self):
        s = _OrcMesh()
        s.n_nodes, s.xy, s.n_elem = self.n_nodes, _d(self.xy), self.n_elem
        s.conn, s.elem_mat, s.is_cut = _i(self.conn), _i(self.elem_mat), _i(self.is_cut)
        s.enr_ptr, s.enr = _i(self.enr_ptr), _i(self.enr)
        s.child_ptr, s.child_nodes_ptr, s.child_nodes = _i(self.child_ptr), _i(self.child_nodes_ptr), _i(self.child_nodes)
        s.child_mat, s.coh_ptr, s.coh_nodes = _i(self.child_mat), _i(self.coh_ptr), _i(self.coh_nodes)
        s.n_mat, s.mat_E, s.mat_nu = self.mat_E.size, _d(self.mat_E), _d(self.mat_nu)
        s.plane_strain, s.coh_law = self.plane_strain, self.coh_law
        for k in range(5):
            s.coh_p[k] = self.coh_p[k]
        return s

    def pattern(self):
        if self._pattern is None:
            s = self._struct()
            rp = np.zeros(2 * self.n_nodes + 1, np.int32)
            nnz = lib().orc_pattern(C.byref(s), _i(rp), None)
            col = np.zeros(nnz, np.int32)
            lib().orc_pattern(C.byref(s), _i(rp), _i(col))
            self._pattern = (rp, col)
        return self._pattern

    def assemble(self, u=None, dt=0.0, isv_c=None, want_K=True, want_f=False):
        """Returns (K as scipy CSR or None, f_int or None, isv_trial)."""
        import scipy.sparse as sp
        rp, col = self.pattern()
        val = np.zeros(col.size)
        nd = 2 * self.n_nodes
        u = np.zeros(nd) if u is None else np.ascontiguousarray(u, dtype=np.float64)
        f = np.zeros(nd)
        nq = max(self.n_coh_qp, 1)
        isv_c = np.zeros(nq) if isv_c is None else np.ascontiguousarray(isv_c, dtype=np.float64)
        isv_t = np.zeros(nq)
        s = self._struct()
        rc = lib().orc_assemble(C.byref(s), _i(rp), _i(col), _d(val), _d(u), float(dt), _d(isv_c), _d(isv_t), _d(f),
                                int(want_K), int(want_f))
        if rc != 0:
            raise RuntimeError(f"oracle geometry error {rc} (negative Jacobian or bad inverse map)")
        K = sp.csr_matrix((val, col, rp), shape=(nd, nd)) if want_K else None
        return K, (f if want_f else None), isv_t[: self.n_coh_qp]


# ---------------------------------------------------------------------------
# adapters
# ---------------------------------------------------------------------------

def from_reference(rec: dict, coh_law=0, coh_p=(0, 0, 0, 0)) -> OracleMesh:
    """Oracle mesh from the reference's own dump (oracle/refio.run)."""
    xy = np.concatenate([rec["mesh.node_xy"], rec["mesh.enr_xy"]])
    nreg = rec["mesh.node_xy"].size // 2
    ne = rec["mesh.elem_mat"].size
    ep, ee = rec["mesh.cut_enr_ptr"], rec["mesh.cut_enr"]
    cp, cnp, cn, cm = rec["mesh.child_ptr"], rec["mesh.child_nodes_ptr"], rec["mesh.child_nodes"], rec["mesh.child_mat"]
    hp, hn = rec["mesh.coh_ptr"], rec["mesh.coh_nodes"]
    enr, ch, chm, coh = {}, {}, {}, {}
    for e in np.nonzero(rec["mesh.is_cut"])[0]:
        enr[e] = [int(v) + nreg for v in ee[ep[e]:ep[e + 1]]]
        ch[e] = [list(cn[cnp[c]:cnp[c + 1]]) for c in range(cp[e], cp[e + 1])]
        chm[e] = [int(cm[c]) for c in range(cp[e], cp[e + 1])]
        coh[e] = [list(hn[4 * k:4 * k + 4]) for k in range(hp[e], hp[e + 1])]
    E = rec["mesh.mat_E"]
    nu = rec["mesh.mat_nu"]
    ref_dof = np.concatenate([rec["dof.node"], rec["dof.enr"]])
    return OracleMesh(xy, rec["mesh.conn"], rec["mesh.elem_mat"], rec["mesh.is_cut"], enr, ch, chm, coh, E, nu,
                      True, coh_law, coh_p, ref_dof=ref_dof, n_free=int(rec["dof.n_free"][0]))


def from_product(export: dict, templates: np.ndarray, rve) -> OracleMesh:
    """Oracle mesh from the product's host mesh export plus its template
    table (pg_template_table layout: 80 int32 per template)."""
    nreg = export["n_regular_nodes"]
    enr, ch, chm, coh = {}, {}, {}, {}
    for c, e in enumerate(export["cut_elem"]):
        T = templates[export["cut_tmpl"][c]]
        n_enr, n_child, n_coh = T[1], T[2], T[3]
        enr[e] = [int(v) for v in export["cut_enr"][c][:n_enr]]
        ch[e] = [list(T[24 + 6 * k: 24 + 6 * k + T[16 + k]]) for k in range(n_child)]
        chm[e] = [int(export["cut_child_mat"][c][k]) for k in range(n_child)]
        coh[e] = [list(T[48 + 4 * k: 48 + 4 * k + 4]) for k in range(n_coh)]
    E = np.array([m[0] for m in rve.materials])
    nu = np.array([m[1] for m in rve.materials])
    return OracleMesh(export["xy"], export["conn"], export["elem_mat"], (export["elem_cut"] >= 0).astype(np.int32),
                      enr, ch, chm, coh, E, nu, rve.plane_strain, rve.coh_law, rve.coh_params,
                      ref_dof=export["ref_dof"], n_free=export["n_free"])


# ---------------------------------------------------------------------------
# reference ordering and solves
# ---------------------------------------------------------------------------

def to_reference_blocks(K, ref_dof, n_free):
    """Permute a node-major DOF matrix into the reference's numbering and
    split it into (K_ff, K_fp, K_pf, K_pp)."""
    import scipy.sparse as sp
    n = K.shape[0]
    P = sp.csr_matrix((np.ones(n), (ref_dof, np.arange(n))), shape=(n, n))
    Kr = (P @ K @ P.T).tocsr()
    f = n_free
    return Kr[:f, :f], Kr[:f, f:], Kr[f:, :f], Kr[f:, f:]


def reference_matrix(rec):
    """The reference's assembled K in its own DOF numbering (full matrix)."""
    import scipy.sparse as sp
    import refio  # noqa: F401 (oracle-local)
    blocks = [refio_csr(rec, n) for n in ("K.ff", "K.fp", "K.pf", "K.pp")]
    return sp.bmat([[blocks[0], blocks[1]], [blocks[2], blocks[3]]]).tocsr()


def refio_csr(rec, name):
    import scipy.sparse as sp
    m, n = rec[name + ".shape"]
    return sp.csr_matrix((rec[name + ".val"], rec[name + ".col"], rec[name + ".rowptr"]), shape=(m, n))


def solve_linear(K, fixed, ubar, t_frac=1.0):
    """Direct solve of K_ff u_f = -K_fp u_p (node-major DOFs), returning u."""
    import scipy.sparse.linalg as sla
    fixed = np.asarray(fixed, bool)
    free = ~fixed
    u = np.zeros(K.shape[0])
    u[fixed] = t_frac * np.asarray(ubar)[fixed]
    Kff = K[free][:, free].tocsc()
    rhs = -(K[free][:, fixed] @ u[fixed])
    u[free] = sla.spsolve(Kff, rhs)
    return u


def tri3_K(xy, E, nu, plane_strain=True):
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    Ke = np.zeros(36)
    lib().orc_tri3_K(_d(xy), E, nu, int(plane_strain), _d(Ke))
    return Ke.reshape(6, 6)


def cohesive_law(law, params, dt, dmax, delta):
    p = np.zeros(5)
    p[:len(params)] = params
    d = np.ascontiguousarray(delta, dtype=np.float64).copy()
    t = np.zeros(2)
    Dc = np.zeros(4)
    dm = C.c_double()
    lib().orc_cohesive_law(int(law), _d(p), float(dt), float(dmax), _d(d), _d(t), _d(Dc), C.byref(dm))
    return t, Dc.reshape(2, 2), dm.value


def newton_load_step(om: "OracleMesh", U, fixed, ubar, t_frac, dt, isv_c, rtol=1e-8, max_it=50):
    """The reference's SNES Newton step restated on the CPU (direct solves,
    backtracking on 0.5||r||^2 with sufficient decrease 1e-4).  Returns
    (U, isv_trial, iterations, ||r0||, ||r||)."""
    import scipy.sparse.linalg as sla
    fixed = np.asarray(fixed, bool)
    free = ~fixed
    U = np.array(U, dtype=np.float64)
    U[fixed] = t_frac * np.asarray(ubar)[fixed]
    _, f, isv_t = om.assemble(u=U, dt=dt, isv_c=isv_c, want_K=False, want_f=True)
    r = f.copy(); r[fixed] = 0.0
    r0 = np.linalg.norm(r)
    rn = r0
    it = 0
    while it < max_it and rn > rtol * r0:
        K, _, _ = om.assemble(u=U, dt=dt, isv_c=isv_c, want_K=True, want_f=False)
        d = np.zeros_like(U)
        d[free] = sla.spsolve(K[free][:, free].tocsc(), -r[free])
        lam = 1.0
        for _ in range(12):
            Ut = U + lam * d
            _, ft, it_t = om.assemble(u=Ut, dt=dt, isv_c=isv_c, want_K=False, want_f=True)
            rt = ft.copy(); rt[fixed] = 0.0
            if np.linalg.norm(rt) ** 2 <= (1 - 2e-4 * lam) * rn ** 2:
                break
            lam *= 0.5
        U, r, isv_t = Ut, rt, it_t
        rn = np.linalg.norm(r)
        it += 1
    return U, isv_t, it, r0, rn
