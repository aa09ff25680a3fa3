"""Generate the golden fixtures in tests/golden/ by running the compiled camille
reference (oracle/_ref/camille_ref, built by oracle/build_ref.py from the
reference's own sources with oracle patches P1-P3).

The reference ships no tests, golden vectors or known-answer fixtures, so these
outputs of the reference itself pin the oracle and the CUDA path. Each fixture
holds, for one small workload: setup products (metrics, Jacobian, mean
gradients, sponge strength), one right-hand side, one filter application, the
FIX_CFL time step of the first step, and the state after 1 and after `steps`
FIX_DT steps.

Usage: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from camille_b200 import cases  # noqa: E402
from oracle import run_ref  # noqa: E402

WORKLOADS = {
    # 2-D quiescent pulse with four sponges: the 256^2 workload's spacing (100/255) and
    # sponge constants on a 48^2 block (a coarser spacing makes the sponge's sigma*dt
    # leave RK4's stability region, in the reference as well)
    "pulse2d_48": lambda: cases.pulse2d(n=48, length=47 * 100.0 / 255.0, sponge=8, nsteps=20),
    # 3-D curvilinear, Mach 0.5, closures only (the 256^3 workload at 16^3)
    "curvi3d_16": lambda: cases.curvi3d(n=16, seed=2, npulses=8, nsteps=5, halfwidth=2.0),
    # 2-D shear layer over a bumped slip wall, Neumann top, sponges at both x ends: the
    # boundary conditions and every non-uniform mean term (rho'/rho_bar included)
    "shear2d_40x32": lambda: cases.shear2d(nx=40, ny=32, nsteps=20),
    # 3-D curvilinear block with a slip wall, a Neumann face and a mean shear
    "wall3d_14": lambda: cases.wall3d(n=14, nsteps=4),
    # 2-D acoustic plane wave: harmonic-wave Dirichlet face, centerline, all-zero face,
    # Neumann face and a sponge relaxing toward the wave
    "waves2d_40x32": lambda: cases.waves2d(nx=40, ny=32, nsteps=20),
    # 3-D quarter round jet: Gaussian entropy wave face and sponge, two centerlines, Neumann
    # faces, an ambient sponge
    "jet3d_14": lambda: cases.jet3d(n=14, nsteps=4),
    # axisymmetric round jet: the 1/r pressure term, the axis centerline, a sheared mean
    "axisym2d_48x32": lambda: cases.axisym2d(nx=48, nr=32, nsteps=20),
    # PHYSICAL_MODEL = LEE_SCALAR: two passive scalars on the shear layer (slip wall, Neumann,
    # sponges, non-uniform mean) and one on the 3-D wall block
    "scalar2d_40x32": lambda: cases.with_scalars(cases.shear2d(nx=40, ny=32, nsteps=20), n=2),
    "scalar3d_14": lambda: cases.with_scalars(cases.wall3d(n=14, nsteps=4), n=1, seed=22),
}

# Two-block overset workloads (run on one reference rank per block).
OVERSET_WORKLOADS = {
    # the cylinder workload at 64^2 + 72x24: hole cut, fringes, O-grid seam, slip wall,
    # sponges, shear layer, monopole, and a pulse that crosses the overlap
    "cylinder2d_64": lambda: cases.cylinder2d(nb=64, length=16.0, ntheta=72, nr=24, r_out=3.0, first_cell=0.05,
                                              r_cut=1.0, sponge=4, nsteps=40, pulse=(1.8, 0.6, 1e-3, 0.5)),
    # one block with hand-set holes and self-donated receivers: every hole-closure branch of
    # iblank_correction (a hole after fluid, after a receiver, after a hole; fluid and receivers
    # after a hole; holes at line starts and ends) along every direction, in 2-D and 3-D
    "holes2d": lambda: cases.holes(2, nsteps=12),
    "holes3d": lambda: cases.holes(3, nsteps=8),
    # two passive scalars through the cylinder layout's hole cut, fringes and seam
    "scalar_cylinder2d_64": lambda: cases.with_scalars(
        cases.cylinder2d(nb=64, length=16.0, ntheta=72, nr=24, r_out=3.0, first_cell=0.05, r_cut=1.0, sponge=4,
                         nsteps=40, pulse=(1.8, 0.6, 1e-3, 0.5)), n=2, seed=23),
}


def make(name: str) -> str:
    case = WORKLOADS[name]()
    nd = case.num_dim
    nv = 5 + case.num_scalars
    setup = run_ref.assemble(case, run_ref.run(case, mode="setup")["ranks"])[0]
    rhs = run_ref.assemble(case, run_ref.run(case, mode="rhs")["ranks"])[0]
    filt = run_ref.assemble(case, run_ref.run(case, mode="filter")["ranks"])[0]
    first = run_ref.run(case, mode="run", nsteps=1, dt=None)
    dt = float(first["result"]["dt"])
    step1 = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=1, dt=dt)["ranks"])[0]
    stepn = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=case.nsteps, dt=dt)["ranks"])[0]
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(
        out,
        metrics=setup[0:9], jacobian=setup[9], mean_gradient=setup[12:12 + nv * nd],
        sponge=setup[12 + nv * nd + 4], rhs=rhs, filter=filt, dt=np.float64(dt),
        step1=step1, stepn=stepn, nsteps=np.int64(case.nsteps))
    return out


def make_overset(name: str) -> str:
    """Per block: iblank, the donor and receiver maps the reference holds, one RHS, the
    FIX_CFL dt, and the state after 1 and after `steps` FIX_DT steps."""
    case = OVERSET_WORKLOADS[name]()
    nb = len(case.blocks)
    ovs = run_ref.run(case, mode="overset", nprocs=nb)["ranks"]
    rhs = run_ref.assemble(case, run_ref.run(case, mode="rhs", nprocs=nb)["ranks"])
    first = run_ref.run(case, mode="run", nsteps=1, dt=None, nprocs=nb)
    dt = float(first["result"]["dt"])
    step1 = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=1, dt=dt, nprocs=nb)["ranks"])
    stepn = run_ref.assemble(case, run_ref.run(case, mode="run", nsteps=case.nsteps, dt=dt, nprocs=nb)["ranks"])
    arrays = {"dt": np.float64(dt), "nsteps": np.int64(case.nsteps)}
    for r in ovs:
        b = r["overset"]["block"]
        arrays[f"iblank_{b}"] = r["fields"][0]
        arrays[f"donor_l0_{b}"] = r["overset"]["donor_l0"]
        arrays[f"weights_{b}"] = r["overset"]["weights"]
        arrays[f"recv_l0_{b}"] = r["overset"]["recv_l0"]
    for b in range(nb):
        arrays[f"rhs_{b}"] = rhs[b]
        arrays[f"step1_{b}"] = step1[b]
        arrays[f"stepn_{b}"] = stepn[b]
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, **arrays)
    return out


if __name__ == "__main__":
    if not run_ref.available():
        sys.exit("build the reference first: python oracle/build_ref.py")
    for n in (sys.argv[1:] or list(WORKLOADS) + list(OVERSET_WORKLOADS)):
        print(make_overset(n) if n in OVERSET_WORKLOADS else make(n))
