"""Run the compiled camille reference (oracle/_ref/camille_ref) on a Case.

Test infrastructure only: used by tests/golden/make_golden.py, the parity
tests and bench.py's CPU-baseline and reference arms, never by the product.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_EXE = os.path.join(HERE, "_ref", "camille_ref")
MPIRUN = os.path.join(HERE, "_ref", "minimpi_run")


def available() -> bool:
    return os.path.isfile(REF_EXE) and os.access(REF_EXE, os.X_OK)


def read_dump(path: str) -> dict:
    with open(path, "rb") as f:
        hdr = np.fromfile(f, "<i4", 16)
        if int(hdr[0]) != 0x4C454532:
            raise ValueError(f"{path}: bad oracle dump magic")
        td = np.fromfile(f, "<f8", 2)
        nd = [int(v) for v in hdr[5:8]]
        n = nd[0] * nd[1] * nd[2]
        nf = int(hdr[8])
        data = np.fromfile(f, "<f8", nf * n).reshape(nf, nd[2], nd[1], nd[0])
    return {"block": int(hdr[1]), "offset": [int(v) for v in hdr[2:5]], "dims": nd,
            "owned": ([int(v) for v in hdr[10:13]], [int(v) for v in hdr[13:16]]),
            "step": int(hdr[9]), "time": float(td[0]), "dt": float(td[1]), "fields": data}


def read_ovs(path: str) -> dict:
    """The donor/receiver maps one rank held (ORACLE_MODE=overset of ref_driver.cpp)."""
    with open(path, "rb") as f:
        block, nd = (int(v) for v in np.fromfile(f, "<i4", 2))
        dl0, coeffs = [], []
        for _ in range(nd):
            l0, nc = (int(v) for v in np.fromfile(f, "<i4", 2))
            dl0.append(l0)
            coeffs.append(np.fromfile(f, "<f8", nc))
        nr = int(np.fromfile(f, "<i4", 1)[0])
        rl0 = np.fromfile(f, "<i4", nr)
    return {"block": block, "donor_l0": np.asarray(dl0, np.int64),
            "weights": np.asarray(coeffs) if coeffs else np.zeros((0, 0)),
            "recv_l0": rl0.astype(np.int64)}


def run(case, mode: str = "run", nsteps: Optional[int] = None, dt: Optional[float] = None,
        nprocs: int = 1, step: int = 0, time: float = 0.0, timeout: float = 3600.0,
        workdir: Optional[str] = None, extra_env: Optional[dict] = None) -> dict:
    """Run the reference; returns {'ranks': [dump...], 'result': {...}, 'stdout': str}.

    ``dt=None`` runs FIX_CFL with the case's CFL; otherwise FIX_DT with ``dt``.
    """
    if not available():
        raise FileNotFoundError("oracle/_ref/camille_ref is not built (python oracle/build_ref.py)")
    nsteps = case.nsteps if nsteps is None else nsteps
    tmp = tempfile.TemporaryDirectory(prefix="camille_ref_") if workdir is None else None
    wd = workdir or tmp.name
    try:
        ic = case.write_reference_inputs(wd, dt, nsteps, step=step, time=time)
        env = dict(os.environ)
        env["ORACLE_MODE"] = mode
        env["ORACLE_DUMP"] = os.path.join(wd, "dump")
        env["ORACLE_NO_WRITE"] = "1"
        env.pop("ORACLE_MONOPOLE", None)
        if case.monopole is not None:
            env["ORACLE_MONOPOLE"] = ",".join(repr(float(v)) for v in case.monopole)
        if extra_env:
            env.update(extra_env)
        cmd = [REF_EXE, ic]
        if nprocs > 1:
            cmd = [MPIRUN, "-n", str(nprocs), "-t", str(int(timeout))] + cmd
        p = subprocess.run(cmd, cwd=wd, env=env, capture_output=True, text=True, errors="replace",
                           timeout=timeout)
        out = p.stdout
        if p.returncode != 0 or "ORACLE_OK" not in out:
            tail = (out[-3000:] + "\n" + p.stderr[-3000:])
            raise RuntimeError(f"reference run failed (rc={p.returncode}):\n{tail}")
        result = {}
        for line in out.splitlines():
            if line.startswith("ORACLE_RESULT ") or line.startswith("ORACLE_SETUP "):
                result.update(json.loads(line.split(" ", 1)[1]))
        ranks = [read_dump(os.path.join(wd, f"dump.{r}.bin")) for r in range(nprocs)]
        if mode == "overset":
            for r, d in enumerate(ranks):
                d["overset"] = read_ovs(os.path.join(wd, f"dump.{r}.ovs"))
        return {"ranks": ranks, "result": result, "stdout": out}
    finally:
        if tmp is not None:
            tmp.cleanup()


def assemble(case, ranks: list[dict]) -> list[np.ndarray]:
    """Stitch per-rank dumps back into one (nf, nz, ny, nx) array per block."""
    out = []
    for b, blk in enumerate(case.blocks):
        nx, ny, nz = blk.dims
        parts = [r for r in ranks if r["block"] == b]
        nf = parts[0]["fields"].shape[0]
        arr = np.full((nf, nz, ny, nx), np.nan)
        for r in parts:
            # only the points the rank owns: its ghost cells are not time-advanced
            (i0, j0, k0), (i1, j1, k1) = r["owned"]
            ox, oy, oz = r["offset"]
            arr[:, oz + k0:oz + k1 + 1, oy + j0:oy + j1 + 1, ox + i0:ox + i1 + 1] = \
                r["fields"][:, k0:k1 + 1, j0:j1 + 1, i0:i1 + 1]
        out.append(arr)
    return out
