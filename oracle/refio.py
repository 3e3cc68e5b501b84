"""Reader/runner for the reference oracle driver (oracle/ref_driver.cpp).

Test infrastructure only: the product never imports this module.  The driver
is the reference (PIGFEM 4.6.1) built from its own sources against the
single-rank shim; this module writes its config, runs it and parses the flat
record file it emits into a dict of numpy arrays.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVER = os.path.join(HERE, "_ref", "pigfem_ref_driver")
# the same driver with the B200 library's solver below the reference's Problem
# (integration/solver_gpu.h; `make -f oracle/Makefile.ref dropin`)
DROPIN_DRIVER = os.path.join(HERE, "_ref", "pigfem_gpu_dropin")


def driver_available() -> bool:
    return os.path.isfile(DRIVER) and os.access(DRIVER, os.X_OK)


def read_records(path: str) -> dict:
    out = {}
    with open(path, "rb") as f:
        data = f.read()
    off = 0
    while off < len(data):
        (nl,) = struct.unpack_from("<i", data, off)
        off += 4
        name = data[off:off + nl].decode()
        off += nl
        dt = chr(data[off])
        off += 1
        (count,) = struct.unpack_from("<q", data, off)
        off += 8
        dtype = {"d": np.float64, "i": np.int32, "q": np.int64}[dt]
        nbytes = count * np.dtype(dtype).itemsize
        out[name] = np.frombuffer(data, dtype=dtype, count=count, offset=off).copy()
        off += nbytes
    return out


def write_config(path: str, cfg: dict) -> None:
    lines = []
    for k, v in cfg.items():
        if k == "inclusions":
            for inc in v:
                lines.append("inc %.17g %.17g %.17g %.17g %.17g" % tuple(inc))
        elif k == "sens":
            for inc, name in v:
                lines.append(f"sens {int(inc)} {name}")
        else:
            lines.append(f"{k} {v}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def run(cfg: dict, timeout: float = 600.0, driver: str = None) -> dict:
    """Run the reference on ``cfg`` and return its records.

    cfg keys: nx, ny, x0, x1, y0, y1, E_matrix, nu_matrix, plane_strain,
    strain, problem ('linear'|'cohesive'), inclusions [(cx, cy, r, E, nu)],
    coh_sigma, coh_delta, coh_beta, coh_visc, T_final, max_dt, min_dt,
    max_iter, assemble_repeats, dump_K, snes_rtol, snes_stol, sens [(inclusion,
    "X"|"Y"|"R")] (shape sensitivities of the right-edge load); write_vtk and
    write_openings (True: the reference's Writer_ASCII_VTK file and
    WriterCohesiveOpenings CSV of the final state come back as the bytes of
    records "vtk.text" and "openings.text").
    """
    driver = driver or DRIVER
    if not os.path.exists(driver):
        raise FileNotFoundError(f"reference driver not built: {driver}")
    cfg = dict(cfg)
    want_vtk = bool(cfg.pop("write_vtk", False))
    want_open = bool(cfg.pop("write_openings", False))
    with tempfile.TemporaryDirectory() as td:
        cfg_path = os.path.join(td, "cfg.txt")
        out_path = os.path.join(td, "out.bin")
        # The reference puts its output folder under ./Output (Options.cpp:208-238).
        os.makedirs(os.path.join(td, "Output"))
        texts = {}
        if want_vtk:
            texts["vtk.text"] = cfg["vtk_out"] = os.path.join(td, "final.vtk")
        if want_open:
            texts["openings.text"] = cfg["openings_out"] = os.path.join(td, "openings.csv")
        write_config(cfg_path, cfg)
        proc = subprocess.run([driver, cfg_path, out_path, "Output/run"], cwd=td,
                              capture_output=True, text=True, timeout=timeout)
        if proc.returncode != 0 or not os.path.exists(out_path):
            raise RuntimeError(f"reference driver failed rc={proc.returncode}\n"
                               f"{proc.stdout[-3000:]}\n{proc.stderr[-3000:]}")
        rec = read_records(out_path)
        for key, path in texts.items():
            with open(path, "rb") as f:
                rec[key] = np.frombuffer(f.read(), dtype=np.uint8).copy()
        rec["_stdout"] = proc.stdout
        rec["_stderr"] = proc.stderr
        return rec


def csr(rec: dict, name: str):
    import scipy.sparse as sp
    m, n = rec[name + ".shape"]
    return sp.csr_matrix((rec[name + ".val"], rec[name + ".col"], rec[name + ".rowptr"]), shape=(m, n))
