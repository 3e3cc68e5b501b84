"""Generates the golden fixtures in tests/golden/ by running the REFERENCE
(PIGFEM 4.6.1, built from its own sources by oracle/Makefile.ref into
oracle/_ref/) through its own Problem API (oracle/ref_driver.cpp).

Run in a container that has the reference mounted and oracle/_ref built:
    make -f oracle/Makefile.ref -j8
    python tests/golden/make_golden.py

Fixtures (numpy .npz):
  linear_8x8.npz      one centred circle r=0.25 on 8x8 (the config-0 geometry, coarse)
  linear_cfg0.npz     config 0: 64x64, r=0.25, E 3.0/70 GPa, nu 0.35/0.2, 1% strain
  linear_3inc.npz     40x40, three circles, two inclusion materials; contains a
                      node on an interface that escapes the node-moving rule
                      (a zero-area child element)
  sensitivity_3inc.npz   32x32, three circles: f (the right edge's mean x
                      reaction) and df/d(x_c, y_c, r) of every inclusion from the
                      reference's SensitivityAdjoint + SensitivityRightLoad
  sensitivity_close.npz  40x40, two circles 0.02 apart (elements cut by both)
  cohesive_16x16.npz  Ortiz-Pandolfi cohesive interface, four load steps from
                      four prefix-consistent runs (committed state per step),
                      each Newton solve converged to SNES rtol 1e-12 (stol off)
                      instead of PETSc's default 1e-8, so that the trajectory
                      itself is accurate to well below the parity bounds
Each holds the reference's enriched mesh, DOF numbering, K_ff/K_fp/K_pf/K_pp
(linear), the solution, (linear) the strain, stress and J W at every
volumetric quadrature point (Problem::compute_stress_strain), and (cohesive)
the internal force and delta_max; and the text of the files the reference's
writers make of the final state: the legacy VTK file (Writer_ASCII_VTK, all
fixtures) and the cohesive openings CSV (WriterCohesiveOpenings, cohesive).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refio  # noqa: E402

KEEP = ("mesh.", "dof.", "K.", "U.", "F.", "Pint.", "isv.", "snes.", "qp.", "vtk.", "openings.", "sens.")


def save(name: str, rec: dict, extra: dict | None = None) -> None:
    out = {k: v for k, v in rec.items() if k.startswith(KEEP)}
    if extra:
        out.update(extra)
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KB)")


def main() -> None:
    if not refio.driver_available():
        raise SystemExit("build the reference first: make -f oracle/Makefile.ref -j8")
    lin = dict(E_matrix=3000.0, nu_matrix=0.35, strain=0.01, problem="linear", write_vtk=True)
    r = refio.run(dict(lin, nx=8, ny=8, inclusions=[(0.5, 0.5, 0.25, 70000.0, 0.2)]))
    save("linear_8x8.npz", r, {"cfg.nx": np.array([8]), "cfg.inc": np.array([[0.5, 0.5, 0.25, 70000.0, 0.2]])})
    r = refio.run(dict(lin, nx=64, ny=64, inclusions=[(0.5, 0.5, 0.25, 70000.0, 0.2)]))
    save("linear_cfg0.npz", r, {"cfg.nx": np.array([64]), "cfg.inc": np.array([[0.5, 0.5, 0.25, 70000.0, 0.2]])})
    incs = [(0.3, 0.3, 0.12, 70000.0, 0.2), (0.7, 0.62, 0.2, 20000.0, 0.3), (0.3, 0.75, 0.1, 70000.0, 0.2)]
    r = refio.run(dict(lin, nx=40, ny=40, inclusions=incs))
    save("linear_3inc.npz", r, {"cfg.nx": np.array([40]), "cfg.inc": np.array(incs)})

    # shape sensitivities of the right-edge load (SensitivityAdjoint with
    # SensitivityRightLoad) for every centre coordinate and radius
    for name, nx, sincs in (
            ("sensitivity_3inc.npz", 32, [(0.3, 0.35, 0.16, 70000.0, 0.2), (0.7, 0.4, 0.13, 70000.0, 0.2),
                                          (0.45, 0.75, 0.15, 20000.0, 0.3)]),
            ("sensitivity_close.npz", 40, [(0.3, 0.5, 0.2, 70000.0, 0.2), (0.72, 0.5, 0.2, 20000.0, 0.3)])):
        params = [(i, k) for i in range(len(sincs)) for k in ("X", "Y", "R")]
        r = refio.run(dict(lin, nx=nx, ny=nx, inclusions=sincs, dump_K=0, write_vtk=False, sens=params))
        assert int(r["sens.adjoint"][0]) == 1
        save(name, r, {"cfg.nx": np.array([nx]), "cfg.inc": np.array(sincs),
                       "cfg.sens_inc": np.array([p[0] for p in params], np.int32),
                       "cfg.sens_kind": np.array(["XYR".index(p[1]) for p in params], np.int32)})

    # cohesive: step k of a run with T_final = k*dt and strain = k*0.0025 has the
    # same load history as the first k steps of any longer run of this family
    base = dict(nx=16, ny=16, E_matrix=3000.0, nu_matrix=0.35, problem="cohesive",
                inclusions=[(0.5, 0.5, 0.25, 70000.0, 0.2)], coh_sigma=10.0, coh_delta=1.5e-4, coh_beta=1.0,
                coh_visc=0.5, min_dt=1e-6, max_iter=40, snes_rtol=1e-12, snes_stol=0.0)
    dt = 0.1
    steps = {}
    for k in range(1, 5):
        rk = refio.run(dict(base, T_final=dt * k, max_dt=dt, strain=0.0025 * k, dump_K=0,
                            write_vtk=(k == 4), write_openings=(k == 4)))
        for key in ("U.f", "U.p", "Pint.f", "Pint.p", "isv.delta_max"):
            steps[f"step{k}.{key}"] = rk[key]
        steps[f"step{k}.snes.iterations"] = rk["snes.iterations"]
        last = rk
    save("cohesive_16x16.npz", last, dict(steps, **{
        "cfg.nx": np.array([16]), "cfg.inc": np.array([[0.5, 0.5, 0.25, 70000.0, 0.2]]),
        "cfg.coh": np.array([10.0, 1.5e-4, 1.0, 0.5]), "cfg.dt": np.array([dt]), "cfg.strain_per_step": np.array([0.0025]),
        "cfg.nsteps": np.array([4]), "cfg.snes_rtol": np.array([1e-12])}))


if __name__ == "__main__":
    main()
