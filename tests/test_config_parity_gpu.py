"""Parity at the sizes and step counts of the benchmark workloads, not only on small cases.

- 2-D pulse, 256^2 on [-50,50]^2, quiescent mean, 20-cell sponges, RK4 at the FIX_CFL 0.5 time
  step (the plain FP64 configuration): the CUDA FP64 path against the live compiled reference
  (``oracle/_ref``, 8 MPI ranks, DECOMP_1D) and the oracle, within 1e-12 relative L2 after one
  step and within 1e-10 after 1000 steps.
- The two-block overset layout at its full size (512^2 background on [-40,40]^2 + a 384x96
  O-grid, first cell 0.005, shear-layer mean, monopole at (2,0)): the receiver/donor maps the GPU
  holds equal, bit for bit, the maps the compiled reference reads from the same Overture file
  (``overset::receiverCells`` / ``donorCells``); FP64 states against the oracle within 1e-12
  after one step and within 1e-10 after 200 steps.
- The 3-D curvilinear mapping (x = xi + 0.1 sin(2 pi eta/L) sin(2 pi zeta/L), cyclic), Mach 0.5,
  8 seeded pulses, with the n/16-cell sponge frame (4 cells), at 64^3: FP64 against the oracle
  within 1e-12 after one step and within 1e-10 after 200 steps (the oracle is pinned bit for bit to
  the compiled reference on this mapping at 16^3 and 20^3).

The FP32-compensated form is compared with the FP64 oracle on each of them (p' relative L2
within 1e-5); the measured errors are printed (``pytest -s``).
"""
from __future__ import annotations

import concurrent.futures as cf

import numpy as np
import pytest

from camille_b200 import api, cases
from oracle import run_ref

pytestmark = pytest.mark.gpu

REF_RANKS = 8


def rl2(a, b):
    return api.rel_l2(np.asarray(a), np.asarray(b))


def _config1():
    return cases.pulse2d(n=256, length=100.0, sponge=20, nsteps=1000)


def _config2_64():
    return cases.curvi3d(n=64, nsteps=200, sponge=4)


def _config3():
    return cases.cylinder2d(nsteps=200)


# The live reference runs in a background thread (a subprocess of 8 ranks) while the GPU and the
# oracle work, FIX_DT at the oracle's FIX_CFL time step.
_POOL = cf.ThreadPoolExecutor(max_workers=1)
_REF = {}


def _reference(label, case, dt):
    if label not in _REF:
        def job():
            out = run_ref.run(case, mode="run", nsteps=case.nsteps, dt=dt, nprocs=REF_RANKS, timeout=1200)
            return run_ref.assemble(case, out["ranks"]), out["result"]
        _REF[label] = _POOL.submit(job)
    return _REF[label]


@pytest.fixture(scope="module")
def config1(oracle_lib):
    case = _config1()
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    ref = _reference("config1", case, dt) if run_ref.available() else None
    o.advance(1, dt)
    y1 = o.download(0)[0]
    o.advance(case.nsteps - 1, dt)
    yn, sn, tn = o.download(0)
    return {"case": case, "dt": dt, "step1": y1, "stepn": yn, "sn": sn, "tn": tn, "ref": ref}


def test_config1_fp64_1000_steps(product_lib, config1):
    case, dt = config1["case"], config1["dt"]
    p = api.Solver(product_lib, case)
    assert abs(p.compute_dt() - dt) <= 1e-14 * dt
    p.advance(1, dt)
    e1 = rl2(p.download(0)[0], config1["step1"])
    p.advance(case.nsteps - 1, dt)
    yp, sp, tp = p.download(0)
    en = rl2(yp, config1["stepn"])
    print(f"\nconfig1 256^2 FP64 vs oracle: step 1 {e1:.3e}, step {case.nsteps} {en:.3e}")
    assert (sp, tp) == (config1["sn"], config1["tn"])
    assert e1 <= 1e-12
    assert en <= 1e-10
    if config1["ref"] is not None:
        yr, res = config1["ref"].result()
        assert res["steps"] == case.nsteps
        er = rl2(yp, yr[0])
        eo = rl2(config1["stepn"], yr[0])
        print(f"config1 256^2 FP64 vs the compiled reference ({REF_RANKS} ranks) after {case.nsteps} steps: "
              f"CUDA {er:.3e}, oracle {eo:.3e}")
        assert er <= 1e-10


def test_config1_fp32_compensated_error(product_lib, config1):
    case, dt = config1["case"], config1["dt"]
    p = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    p.advance(case.nsteps, dt)
    err = rl2(p.download(0)[0][4], config1["stepn"][4])
    print(f"\nconfig1 256^2 FP32-compensated p' vs FP64 oracle after {case.nsteps} steps: {err:.3e}")
    assert err <= 1e-5


@pytest.fixture(scope="module")
def config2(oracle_lib):
    case = _config2_64()
    o = api.Solver(oracle_lib, case)
    dt = o.compute_dt()
    o.advance(1, dt)
    y1 = o.download(0)[0]
    o.advance(case.nsteps - 1, dt)
    return {"case": case, "dt": dt, "step1": y1, "stepn": o.download(0)[0]}


def test_config2_mapping_64_fp64_200_steps(product_lib, config2):
    case, dt = config2["case"], config2["dt"]
    p = api.Solver(product_lib, case)
    assert p.info().tma_stage == 1 and p.info().tma_filter == 1
    assert abs(p.compute_dt() - dt) <= 1e-14 * dt
    p.advance(1, dt)
    e1 = rl2(p.download(0)[0], config2["step1"])
    p.advance(case.nsteps - 1, dt)
    yp = p.download(0)[0]
    en = rl2(yp, config2["stepn"])
    print(f"\ncurvilinear 64^3 + sponge frame FP64 vs oracle: step 1 {e1:.3e}, step {case.nsteps} {en:.3e}")
    assert e1 <= 1e-12
    assert en <= 1e-10


def test_config2_mapping_64_fp32_compensated_error(product_lib, config2):
    case, dt = config2["case"], config2["dt"]
    p = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED)
    p.advance(case.nsteps, dt)
    err = rl2(p.download(0)[0][4], config2["stepn"][4])
    print(f"\ncurvilinear 64^3 FP32-compensated p' vs FP64 oracle after {case.nsteps} steps: {err:.3e}")
    assert err <= 1e-5


@pytest.fixture(scope="module")
def config3(oracle_lib, tmp_path_factory):
    case = _config3()
    path = str(tmp_path_factory.mktemp("config3") / "overset.bin")
    case.overset.write(path)
    o = api.Solver(oracle_lib, case, overset_file=path)
    dt = o.compute_dt()
    o.advance(1, dt)
    y1 = [o.download(b)[0] for b in range(2)]
    o.advance(case.nsteps - 1, dt)
    return {"case": case, "path": path, "dt": dt, "step1": y1, "stepn": [o.download(b)[0] for b in range(2)]}


def test_config3_full_layout_maps_are_bit_exact(product_lib, config3):
    """The compiled reference reads the same Overture file on one rank per block."""
    if not run_ref.available():
        pytest.skip("oracle/_ref is not built")
    case = config3["case"]
    ranks = run_ref.run(case, mode="overset", nprocs=len(case.blocks), timeout=600)["ranks"]
    m = api.Solver(product_lib, case, overset_file=config3["path"]).get_overset()
    nrecv = 0
    for r in ranks:
        b = r["overset"]["block"]
        sel = m["donor_block"] == b
        np.testing.assert_array_equal(m["donor_l0"][sel], r["overset"]["donor_l0"])
        np.testing.assert_array_equal(m["weights"][sel], r["overset"]["weights"])
        np.testing.assert_array_equal(m["recv_l0"][m["recv_block"] == b], r["overset"]["recv_l0"])
        nrecv += len(r["overset"]["recv_l0"])
    print(f"\nfull overset layout: {nrecv} receivers, maps bit-exact")
    assert nrecv == len(m["recv_l0"]) and nrecv > 1000


def test_config3_full_layout_fp64_200_steps(product_lib, config3):
    case, dt = config3["case"], config3["dt"]
    p = api.Solver(product_lib, case, overset_file=config3["path"])
    assert abs(p.compute_dt() - dt) <= 1e-14 * dt
    p.advance(1, dt)
    e1 = [rl2(p.download(b)[0], config3["step1"][b]) for b in range(2)]
    p.advance(case.nsteps - 1, dt)
    en = [rl2(p.download(b)[0], config3["stepn"][b]) for b in range(2)]
    print(f"\nfull overset layout FP64 vs oracle: step 1 {e1[0]:.3e}/{e1[1]:.3e}, "
          f"step {case.nsteps} {en[0]:.3e}/{en[1]:.3e} (background/O-grid)")
    assert max(e1) <= 1e-12
    assert max(en) <= 1e-10


def test_config3_full_layout_fp32_compensated_error(product_lib, config3):
    case, dt = config3["case"], config3["dt"]
    p = api.Solver(product_lib, case, precision=api.FP32_COMPENSATED, overset_file=config3["path"])
    p.advance(case.nsteps, dt)
    err = [rl2(p.download(b)[0][4], config3["stepn"][b][4]) for b in range(2)]
    print(f"\nfull overset layout FP32-compensated p' vs FP64 oracle after {case.nsteps} steps: "
          f"{err[0]:.3e}/{err[1]:.3e}")
    assert max(err) <= 1e-5
