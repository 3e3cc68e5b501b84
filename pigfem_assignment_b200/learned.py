"""Learned Newton warm start for cohesive load stepping.

A per-node MLP (16 -> 64 -> 64 -> 16, two outputs used; BF16 tensor-core
kernels with FP32 accumulation, trained by this library's own forward/
backward kernels and Adam) predicts the correction of the linear load
extrapolation of every node's displacement at the start of a load step:

    U_pred = U_n + ratio (U_n - U_{n-1}) + s * MLP(features)

at enrichment nodes and nodes with cohesive damage (elsewhere the linear
extrapolation is kept: in the elastic bulk it is already close, and any
network output there only adds error).

Training data are trajectories the GPU Newton solver itself generates
(features at the start of step n+1, targets from the converged U_{n+1}).
Inside pg_solve_nonlinear (predictor PG_PREDICT_LEARNED) the plain linear
extrapolation is the fallback whenever it starts from the smaller residual,
and the converged Newton residual decides every step's result, so the
network can only change how many iterations a step takes, never what it
converges to.  The reference has no learned component (its predictor keeps
the last converged U_f, src/SolverNonlinear.cpp:254-267).
"""
from __future__ import annotations

import ctypes as C
import time
from typing import List, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .problem import ProblemNonlinearStructural
from .rve import RVE


def _torch():
    import torch
    return torch


class MLP:
    """Handle of a device MLP (pg_mlp)."""

    def __init__(self, device: int = 0, seed: int = 0):
        h = C.c_void_p()
        check(lib.pg_mlp_create(device, seed, C.byref(h)), "pg_mlp_create")
        self.handle = h
        self.device = device

    _destroy = lib.pg_mlp_destroy  # held by the class: usable while the interpreter shuts down

    def close(self):
        if getattr(self, "handle", None):
            self._destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        v = np.zeros(lib.pg_mlp_param_count(), np.float32)
        check(lib.pg_mlp_params(self.handle, v.ctypes.data_as(C.POINTER(C.c_float)), 0))
        return v

    def set_params(self, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, dtype=np.float32)
        check(lib.pg_mlp_params(self.handle, v.ctypes.data_as(C.POINTER(C.c_float)), 1))

    def zero_output_layer(self, bias: float = 0.0) -> None:
        """Output weights to zero and the two used outputs' biases to `bias`:
        the network then starts as the constant y = bias (-1: the linear
        extrapolation of the learned predictor, 0: the quadratic one)."""
        v = self.params()
        v[-(16 * 64 + 16):] = 0.0
        v[-16] = v[-15] = bias
        self.set_params(v)

    def forward(self, X):
        torch = _torch()
        Y = torch.empty((X.shape[0], 2), dtype=torch.float32, device=X.device)
        check(lib.pg_mlp_forward(self.handle, C.c_void_p(X.data_ptr()), X.shape[0], C.c_void_p(Y.data_ptr()), None))
        return Y

    def train(self, X, T, epochs: int = 30, batch: int = 8192, lr: float = 2e-3) -> np.ndarray:
        hist = np.zeros(epochs)
        check(lib.pg_mlp_train(self.handle, C.c_void_p(X.data_ptr()), C.c_void_p(T.data_ptr()), X.shape[0], epochs,
                               batch, lr, hist.ctypes.data_as(C.POINTER(C.c_double))), "pg_mlp_train")
        return hist


def _dev_ptrs(ctx):
    K, U, F, ic, it = (_lib._dp() for _ in range(5))
    check(lib.pg_ctx_device_arrays(ctx.handle, C.byref(K), C.byref(U), C.byref(F), C.byref(ic), C.byref(it)))
    return C.cast(U, C.c_void_p).value


def trajectory_samples(rve: RVE, n_steps: int, n_train_steps: int, keep_fraction: float = 0.0, seed: int = 0,
                       device: int = 0, rtol: float = 1e-8, newton: dict = None
                       ) -> Tuple["object", "object", List[_lib.StepStats]]:
    """Runs the first `n_train_steps` of `n_steps` equal load steps of `rve`
    with the linear predictor and returns (features, targets) of the nodes
    kept, from the third step on (the features need three converged states),
    plus the step records.  A free node is kept with probability
    min(1, (|c| / c_ref)^2), c its quadratic term and c_ref the 99th
    percentile of |c| over the step's free nodes: the plain mean square error
    over the kept nodes then weighs every node as its error (e - g c) weighs
    in the prediction, where y's target is noise for nodes that barely bend.
    A random `keep_fraction` of the others is kept as well.  `newton` holds
    further pg_newton_cfg fields (e.g. the preconditioner)."""
    torch = _torch()
    prob = ProblemNonlinearStructural(rve, device=device)
    prob.init()
    prob.configure(rtol=rtol, n_steps=n_steps, **(newton or {}))
    ctx = prob.ctx
    n_nodes = prob.mesh.info["n_nodes"]
    n_reg = prob.mesh.info["n_regular_nodes"]
    n_qp = max(1, prob.mesh.info["n_cohesive_qp"])
    U_ptr = _dev_ptrs(ctx)
    nd = 2 * n_nodes
    dev = f"cuda:{device}"
    U = [torch.zeros(nd, dtype=torch.float64, device=dev) for _ in range(3)]  # U_n, U_{n-1}, U_{n-2}
    isv_nm1 = torch.zeros(n_qp, dtype=torch.float64, device=dev)
    X = torch.empty((n_nodes, 16), dtype=torch.float32, device=dev)
    T = torch.empty((n_nodes, 2), dtype=torch.float32, device=dev)
    app = (rve.x1 - rve.x0) * rve.strain
    dt = 1.0 / n_steps
    s_inc = app * dt
    rng = np.random.default_rng(seed)
    xs, ts, recs = [], [], []
    for k in range(1, n_train_steps + 1):
        tf = k * dt
        h = _lib.PredHistory(U[0].data_ptr(), U[1].data_ptr(), U[2].data_ptr(), isv_nm1.data_ptr(), dt, dt, dt, tf,
                             s_inc)
        have_hist = k > 2
        if have_hist:
            check(lib.pg_predictor_features(ctx.handle, C.byref(h), C.c_void_p(X.data_ptr())))
        if k > 1:  # linear extrapolation as the step's start
            check(lib.pg_predictor_apply(ctx.handle, C.byref(h), None, 0.0, C.c_void_p(U_ptr)))
        isv_n = torch.from_numpy(np.resize(ctx.isv(committed=True), n_qp)).to(dev)
        st = prob.load_step(tf, dt)
        if st.reason <= 0:
            break
        prob.commit()
        recs.append(st)
        ctx.sync()
        torch.cuda.synchronize()
        U_cur = torch.from_numpy(ctx.vector(0)).to(dev)
        if have_hist:
            check(lib.pg_predictor_targets(ctx.handle, C.byref(h), C.c_void_p(U_cur.data_ptr()),
                                           C.c_void_p(T.data_ptr())))
            ctx.sync()
            Xh = X.cpu().numpy()
            free = (Xh[:, 12] == 0) | (Xh[:, 13] == 0)
            w = (np.hypot(Xh[:, 0], Xh[:, 1]) * np.expm1(Xh[:, 5])) ** 2  # (|c| / s_inc)^2
            pos = w[free & (w > 0)]
            w_ref = np.quantile(pos, 0.99) if pos.size else 1.0
            keep = (rng.random(n_nodes) < np.minimum(1.0, w / max(w_ref, 1e-300))) | (rng.random(n_nodes) < keep_fraction)
            sel = np.nonzero(keep & free)[0]
            xs.append(Xh[sel])
            ts.append(T.cpu().numpy()[sel])
        U[2].copy_(U[1])
        U[1].copy_(U[0])
        U[0].copy_(U_cur)
        isv_nm1.copy_(isv_n)
    ctx.close()
    return (np.concatenate(xs) if xs else np.zeros((0, 16), np.float32),
            np.concatenate(ts) if ts else np.zeros((0, 2), np.float32), recs)


def compare_predictors(rve: RVE, n_steps: int, mlp: MLP = None, device: int = 0, rtol: float = 1e-8,
                       precision: int = _lib.PG_PRECISION_FP64):
    """Load-steps `rve` with the zeroth-order, linear and learned predictors;
    returns {name: dict(newton_its, seconds, ms_per_step, final U norm)}."""
    out = {}
    modes = [("zeroth", _lib.PG_PREDICT_ZEROTH), ("linear", _lib.PG_PREDICT_LINEAR)]
    if mlp is not None:
        modes.append(("learned", _lib.PG_PREDICT_LEARNED))
    for name, mode in modes:
        prob = ProblemNonlinearStructural(rve, device=device)
        prob.init()
        prob.configure(rtol=rtol, n_steps=n_steps, predictor=mode, precision=precision)
        if mode == _lib.PG_PREDICT_LEARNED:
            check(lib.pg_ctx_attach_mlp(prob.ctx.handle, mlp.handle))
        t0 = time.perf_counter()
        recs = prob.solve_problem()
        wall = time.perf_counter() - t0
        u = prob.get_solution()
        out[name] = {
            "steps": len(recs),
            "newton_its": int(sum(r.newton_its for r in recs)),
            "krylov_its": int(sum(r.krylov_its for r in recs)),
            "device_seconds": float(sum(r.seconds for r in recs)),
            "ms_per_step": 1e3 * float(sum(r.seconds for r in recs)) / max(1, len(recs)),
            "wall_seconds": wall,
            "learned_used": int(sum(1 for r in recs if r.predictor_used == _lib.PG_PREDICT_LEARNED)),
            "u_norm": float(np.linalg.norm(u)),
            "max_rel_res": float(max((r.res / r.res0 if r.res0 > 0 else 0.0) for r in recs)) if recs else 0.0,
        }
        if mode == _lib.PG_PREDICT_LEARNED:
            check(lib.pg_ctx_attach_mlp(prob.ctx.handle, None))
        prob.ctx.close()
    return out
