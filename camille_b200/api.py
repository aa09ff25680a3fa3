"""ctypes binding of the C ABI in include/lee_b200.h.

``Library`` binds one shared object exporting that ABI under a symbol prefix:
``lee_`` for this package's CUDA library (camille_b200/liblee_b200.so) and
``orc_`` for the test-only CPU oracle. ``Solver`` drives a :class:`cases.Case`
through the calls in the order a replacement ``solver::solve`` makes them.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import cases as _cases

PKG = os.path.dirname(os.path.abspath(__file__))
PRODUCT_LIB = os.path.join(PKG, "liblee_b200.so")

LEE_OK = 0
LEE_ERR_ARG, LEE_ERR_STATE, LEE_ERR_UNSUPPORTED = 1, 2, 5
ERRORS = {1: "LEE_ERR_ARG", 2: "LEE_ERR_STATE", 3: "LEE_ERR_CUDA", 4: "LEE_ERR_NOMEM",
          5: "LEE_ERR_UNSUPPORTED", 6: "LEE_ERR_NONFINITE", 7: "LEE_ERR_NODEVICE", 8: "LEE_ERR_TIMEOUT"}
FD = {"STANDARD_CENTRAL": 1, "FDO11P": 11}
FILTER = {"NONE": 0, "STANDARD_CENTRAL": 1, "SFO11P": 11}
RK = {"RUNGE_KUTTA2": 2, "RUNGE_KUTTA4": 4}
FP64, FP32_COMPENSATED = 0, 1
SOURCE_DISTRIBUTED = 2
SETUP_METRICS, SETUP_JACOBIAN, SETUP_MEAN_GRADIENT, SETUP_SPONGE = 0, 1, 2, 3
SOURCE_MONOPOLE = 1
SOURCE_JET2D_HARMONIC = 3
WAVE_NONE, WAVE_ACOUSTIC, WAVE_ENTROPY = 0, 1, 2
WAVEFORM_PLANE, WAVEFORM_HOMOGENEOUS, WAVEFORM_GAUSSIAN_ROUNDJET = 0, 1, 2


class LeeConfig(C.Structure):
    _fields_ = [
        ("num_dim", C.c_int), ("num_blocks", C.c_int), ("gamma", C.c_double),
        ("fd_scheme", C.c_int), ("fd_order", C.c_int),
        ("filter_scheme", C.c_int), ("filter_order", C.c_int),
        ("filter_strength", C.c_double), ("filter_blend", C.c_double),
        ("rk_scheme", C.c_int), ("precision", C.c_int),
        ("sponge_order", C.c_int), ("sponge_constant", C.c_double),
        ("device", C.c_int),
    ]


class LeeInfo(C.Structure):
    _fields_ = [("points", C.c_longlong), ("state_vars", C.c_int), ("bytes_per_value", C.c_int),
                ("num_coef_fields", C.c_int), ("device_bytes", C.c_longlong),
                ("tma_stage", C.c_int), ("tma_filter", C.c_int), ("stage_chunk", C.c_int),
                ("filter_chunk", C.c_int), ("batched", C.c_int), ("batch_stage_tile", C.c_int * 2),
                ("batch_filter_tile", C.c_int * 2), ("filter_kernel", C.c_int), ("stage_kernel", C.c_int),
                ("filter_rows", C.c_int), ("increment_step", C.c_int)]


class LeeStats(C.Structure):
    _fields_ = [("advance_ms", C.c_double), ("stage_ms", C.c_double), ("filter_ms", C.c_double),
                ("stage_launches", C.c_longlong), ("filter_launches", C.c_longlong),
                ("kernel_launches", C.c_longlong)]


class LeeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_DP = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)
_PP = C.POINTER(_DP)
_LP = C.POINTER(C.c_longlong)

# name -> (restype, argtypes); the first argument of most is the context pointer.
SIGNATURES = {
    "create": (C.c_int, [C.POINTER(LeeConfig), C.POINTER(C.c_void_p)]),
    "destroy": (None, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "set_block": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _IP]),
    "set_mean": (C.c_int, [C.c_void_p, C.c_int, _PP]),
    "add_boundary": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _IP, _IP, _DP]),
    "set_harmonic_wave": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]),
    "set_axisymmetric": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "set_source": (C.c_int, [C.c_void_p, C.c_int, _DP, C.c_int]),
    "set_block_source": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _DP, C.c_int]),
    "advance_blocks": (C.c_int, [C.c_void_p, C.c_int, _DP]),
    "compute_dt_blocks": (C.c_int, [C.c_void_p, C.c_double, _DP]),
    "set_batch_shapes": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "set_batch_persistent": (C.c_int, [C.c_void_p, C.c_int]),
    "set_overset": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP, _IP, _IP, _IP, _DP, C.c_int, _IP, _IP]),
    "read_overset_file": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    "get_overset": (C.c_int, [C.c_void_p, _IP, _LP, _IP, _LP, _DP]),
    "prepare": (C.c_int, [C.c_void_p]),
    "upload_state": (C.c_int, [C.c_void_p, C.c_int, _PP, C.c_int, C.c_double]),
    "download_state": (C.c_int, [C.c_void_p, C.c_int, _PP, _IP, _DP]),
    "compute_dt": (C.c_int, [C.c_void_p, C.c_double, _DP]),
    "compute_cfl": (C.c_int, [C.c_void_p, C.c_double, _DP]),
    "state_minmax": (C.c_int, [C.c_void_p, _DP, _DP]),
    "advance": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "eval_rhs": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _PP]),
    "apply_filter": (C.c_int, [C.c_void_p]),
    "get_setup": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _DP]),
    "get_info": (C.c_int, [C.c_void_p, C.POINTER(LeeInfo)]),
    "set_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "get_stats": (C.c_int, [C.c_void_p, C.POINTER(LeeStats)]),
    "set_graphs": (C.c_int, [C.c_void_p, C.c_int]),
    "set_finite_check": (C.c_int, [C.c_void_p, C.c_int]),
    "set_block_streams": (C.c_int, [C.c_void_p, C.c_int]),
    "set_increment_step": (C.c_int, [C.c_void_p, C.c_int]),
    "set_batching": (C.c_int, [C.c_void_p, C.c_int]),
    "set_wait_limit": (C.c_int, [C.c_void_p, C.c_double]),
    "set_filter_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "set_stage_kernel": (C.c_int, [C.c_void_p, C.c_int]),
    "set_filter_form": (C.c_int, [C.c_void_p, C.c_int]),
    "set_objective": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _LP, C.c_double]),
    "eval_objective": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _DP]),
    "apply_adjoint": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "adjoint_gradient": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, _DP, _DP, _LP]),
    "set_scalars": (C.c_int, [C.c_void_p, C.c_int]),
    "set_mean_scalars": (C.c_int, [C.c_void_p, C.c_int, _PP]),
    "upload_scalars": (C.c_int, [C.c_void_p, C.c_int, _PP]),
    "download_scalars": (C.c_int, [C.c_void_p, C.c_int, _PP]),
}


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _fields_ptrs(arrs) -> C.Array:
    return (_DP * len(arrs))(*[_dptr(a) for a in arrs])


class Library:
    def __init__(self, path: str, prefix: str):
        if not os.path.isfile(path):
            raise FileNotFoundError(f"{path} is not built")
        self.path = path
        self.prefix = prefix
        self.dll = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(self.dll, prefix + name)
            fn.restype = res
            fn.argtypes = args
            setattr(self, name, fn)


def product_library() -> Library:
    """The CUDA library. Raises if it is not built: there is no CPU fallback."""
    return Library(PRODUCT_LIB, "lee_")


def config_for(case: "_cases.Case", precision: int = FP64, device: int = 0) -> LeeConfig:
    return LeeConfig(
        num_dim=case.num_dim, num_blocks=len(case.blocks), gamma=case.gamma,
        fd_scheme=FD[case.fd_scheme], fd_order=case.fd_order,
        filter_scheme=FILTER[case.filter_scheme], filter_order=case.filter_order,
        filter_strength=case.filter_strength, filter_blend=case.filter_blend,
        rk_scheme=RK[case.rk], precision=precision,
        sponge_order=case.sponge_order, sponge_constant=case.sponge_constant, device=device)


class Solver:
    """A context loaded with one Case: grids, means, boundaries, source and state."""

    def __init__(self, lib: Library, case: "_cases.Case", precision: int = FP64, device: int = 0,
                 upload: bool = True, overset_file: Optional[str] = None, filter_kernel: int = -1,
                 stage_kernel: int = -1, prepare: bool = True, batching: bool = True, filter_form: int = 0):
        """``overset_file``: read the case's overset maps from this Overture-format file
        (lee_read_overset_file) instead of passing the arrays (lee_set_overset).
        ``filter_kernel``: lee_set_filter_kernel (-1/0 scalar, 2/4 vector width);
        ``stage_kernel``: lee_set_stage_kernel (-1 default, 1 or 2 points per thread);
        ``filter_form``: lee_set_filter_form (0 timed, else the scalar fused filter's form 1, 2 or 3).
        ``batching=False``: lee_set_batching(0), every block runs its own kernels;
        ``prepare=False`` stops before lee_prepare (nothing is uploaded)."""
        self.lib = lib
        self.case = case
        self.ctx = C.c_void_p()
        cfg = config_for(case, precision, device)
        rc = lib.create(C.byref(cfg), C.byref(self.ctx))
        if rc != LEE_OK:
            raise LeeError(rc, lib.last_error(None).decode())
        try:
            if case.num_scalars:
                self._chk(lib.set_scalars(self.ctx, case.num_scalars))
            for b, blk in enumerate(case.blocks):
                nx, ny, nz = blk.dims
                xs = [np.ascontiguousarray(a, np.float64) for a in (blk.x, blk.y, blk.z)]
                ib = None
                if blk.iblank is not None:
                    ibarr = np.ascontiguousarray(blk.iblank, np.int32)
                    ib = ibarr.ctypes.data_as(_IP)
                self._chk(lib.set_block(self.ctx, b, nx, ny, nz, *[_dptr(a) for a in xs], ib))
                mean = [np.ascontiguousarray(blk.mean[v], np.float64) for v in range(5)]
                self._chk(lib.set_mean(self.ctx, b, _fields_ptrs(mean)))
                if case.num_scalars:
                    zm = [np.ascontiguousarray(z, np.float64) for z in blk.zmean]
                    self._chk(lib.set_mean_scalars(self.ctx, b, _fields_ptrs(zm)))
            for bd in case.boundaries:
                lo = (C.c_int * 3)(*bd.lo)
                hi = (C.c_int * 3)(*bd.hi)
                sig = None
                if bd.sigma is not None:
                    sarr = np.ascontiguousarray(bd.sigma, np.float64)
                    sig = _dptr(sarr)
                self._chk(lib.add_boundary(self.ctx, bd.block, _cases.BC_TYPES[bd.kind], bd.dir, bd.end,
                                           lo, hi, sig))
            if case.harmonic_wave is not None:
                self._chk(lib.set_harmonic_wave(self.ctx, *case.harmonic_wave.args()))
            if case.axisymmetric:
                self._chk(lib.set_axisymmetric(self.ctx, 1, 0))
            if case.simulation == "CASE_2DJET_WITH_A_HARMONIC_SOURCE":
                self._chk(lib.set_source(self.ctx, SOURCE_JET2D_HARMONIC, None, 0))
            if case.source_monopole() is not None:
                p = np.array(case.source_monopole(), np.float64)
                self._chk(lib.set_source(self.ctx, SOURCE_MONOPOLE, _dptr(p), len(p)))
            for b, blk in enumerate(case.blocks):
                if blk.monopole is not None:
                    p = np.array(blk.monopole, np.float64)
                    self._chk(lib.set_block_source(self.ctx, b, SOURCE_MONOPOLE, _dptr(p), len(p)))
            if case.distributed is not None:
                p = np.ascontiguousarray(case.distributed.params(), np.float64)
                self._chk(lib.set_source(self.ctx, SOURCE_DISTRIBUTED, _dptr(p), len(p)))
            if overset_file is not None:
                self._chk(lib.read_overset_file(self.ctx, overset_file.encode(), case.overset.order))
            elif case.overset is not None:
                o = case.overset
                arrs = [np.ascontiguousarray(a, np.int32) for a in
                        (o.recv_block, o.recv_ijk, o.donor_block, o.donor_ijk, np.asarray(o.width),
                         o.hole_block, o.hole_ijk)]
                w = np.ascontiguousarray(o.weights, np.float64)
                ip = [a.ctypes.data_as(_IP) for a in arrs]
                self._chk(lib.set_overset(self.ctx, o.num_receivers, ip[0], ip[1], ip[2], ip[3], ip[4], _dptr(w),
                                          int(o.hole_block.size), ip[5], ip[6]))
            if filter_kernel != -1:
                self._chk(lib.set_filter_kernel(self.ctx, filter_kernel))
            if stage_kernel != -1:
                self._chk(lib.set_stage_kernel(self.ctx, stage_kernel))
            if filter_form:
                self._chk(lib.set_filter_form(self.ctx, filter_form))
            if not batching:
                self._chk(lib.set_batching(self.ctx, 0))
            if not prepare:
                return
            self._chk(lib.prepare(self.ctx))
            if case.microphones is not None:
                mic = np.ascontiguousarray(case.microphones.l0, np.int64)
                w = case.microphones.weight
                if w is None:
                    w = self.compute_dt()
                self._chk(lib.set_objective(self.ctx, case.microphones.block, len(mic), mic.ctypes.data_as(_LP), w))
            if upload:
                for b, blk in enumerate(case.blocks):
                    self.upload(b, blk.state)
        except Exception:
            self.close()
            raise

    def _chk(self, rc: int) -> None:
        if rc != LEE_OK:
            raise LeeError(rc, self.lib.last_error(self.ctx).decode())

    def close(self) -> None:
        if self.ctx:
            self.lib.destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, b: int, state: np.ndarray, step: int = 0, time: float = 0.0) -> None:
        """The five LEE slots of block b, and with passive scalars the slots after them: a state
        of 5 + n fields uploads both (lee_upload_state, lee_upload_scalars)."""
        f = [np.ascontiguousarray(state[v], np.float64) for v in range(5)]
        self._chk(self.lib.upload_state(self.ctx, b, _fields_ptrs(f), step, time))
        n = self.case.num_scalars
        if n:
            blk = self.case.blocks[b]
            z = state[5:5 + n] if state.shape[0] >= 5 + n else blk.zstate
            zf = [np.ascontiguousarray(z[k], np.float64) for k in range(n)]
            self._chk(self.lib.upload_scalars(self.ctx, b, _fields_ptrs(zf)))

    def download_scalars(self, b: int = 0) -> np.ndarray:
        """The passive scalars Z_k' of block b, (n, nz, ny, nx)."""
        n = self.case.num_scalars
        nx, ny, nz = self.case.blocks[b].dims
        out = np.zeros((n, nz, ny, nx))
        self._chk(self.lib.download_scalars(self.ctx, b, _fields_ptrs([out[k] for k in range(n)])))
        return out

    def download(self, b: int = 0) -> tuple[np.ndarray, int, float]:
        nx, ny, nz = self.case.blocks[b].dims
        out = np.zeros((5, nz, ny, nx))
        ptrs = _fields_ptrs([out[v] for v in range(5)])
        step = C.c_int()
        time = C.c_double()
        self._chk(self.lib.download_state(self.ctx, b, ptrs, C.byref(step), C.byref(time)))
        return out, step.value, time.value

    def compute_dt(self, cfl: Optional[float] = None) -> float:
        dt = C.c_double()
        self._chk(self.lib.compute_dt(self.ctx, self.case.cfl if cfl is None else cfl, C.byref(dt)))
        return dt.value

    def compute_cfl(self, dt: float) -> float:
        out = C.c_double()
        self._chk(self.lib.compute_cfl(self.ctx, dt, C.byref(out)))
        return out.value

    def state_minmax(self) -> tuple[np.ndarray, np.ndarray]:
        mn, mx = np.zeros(5), np.zeros(5)
        self._chk(self.lib.state_minmax(self.ctx, _dptr(mn), _dptr(mx)))
        return mn, mx

    def advance(self, nsteps: int, dt: float) -> None:
        self._chk(self.lib.advance(self.ctx, nsteps, dt))

    def compute_dt_blocks(self, cfl: Optional[float] = None) -> np.ndarray:
        out = np.zeros(len(self.case.blocks), np.float64)
        self._chk(self.lib.compute_dt_blocks(self.ctx, self.case.cfl if cfl is None else cfl, _dptr(out)))
        return out

    def advance_blocks(self, nsteps: int, dts) -> None:
        d = np.ascontiguousarray(dts, np.float64)
        self._chk(self.lib.advance_blocks(self.ctx, nsteps, _dptr(d)))

    def eval_rhs(self, b: int = 0, time: float = 0.0) -> np.ndarray:
        nx, ny, nz = self.case.blocks[b].dims
        out = np.zeros((5, nz, ny, nx))
        self._chk(self.lib.eval_rhs(self.ctx, b, time, _fields_ptrs([out[v] for v in range(5)])))
        return out

    def apply_filter(self) -> None:
        self._chk(self.lib.apply_filter(self.ctx))

    def eval_objective(self, nsteps: int, dt: float) -> float:
        J = C.c_double()
        self._chk(self.lib.eval_objective(self.ctx, nsteps, dt, C.byref(J)))
        return J.value

    def apply_adjoint(self, nsteps: int, dt: float) -> None:
        self._chk(self.lib.apply_adjoint(self.ctx, nsteps, dt))

    def adjoint_gradient(self, nsteps: int, dt: float, checkpoint_every: int = 100,
                         recompute: bool = True) -> tuple[float, np.ndarray, int]:
        """(J, dJ/d amplitudes, recomputed trace values that differ from the first pass)."""
        d = self.case.distributed
        grad = np.zeros(d.amplitudes.size, np.float64)
        J = C.c_double()
        mism = C.c_longlong()
        self._chk(self.lib.adjoint_gradient(self.ctx, nsteps, dt, checkpoint_every, 1 if recompute else 0,
                                            C.byref(J), _dptr(grad), C.byref(mism)))
        return J.value, grad.reshape(d.amplitudes.shape), mism.value

    def get_overset(self) -> dict:
        """The donor maps the context holds: receiver/donor blocks, linear indices and the
        normalised weights."""
        o = self.case.overset
        n = o.num_receivers if o is not None else 0
        W = int(np.prod(o.width)) if o is not None else 1
        rb = np.zeros(n, np.int32); db = np.zeros(n, np.int32)
        rl = np.zeros(n, np.int64); dl = np.zeros(n, np.int64)
        wt = np.zeros((n, W), np.float64)
        self._chk(self.lib.get_overset(self.ctx, rb.ctypes.data_as(_IP), rl.ctypes.data_as(_LP),
                                       db.ctypes.data_as(_IP), dl.ctypes.data_as(_LP), _dptr(wt)))
        return {"recv_block": rb, "recv_l0": rl, "donor_block": db, "donor_l0": dl, "weights": wt}

    def get_setup(self, b: int, what: int) -> np.ndarray:
        nx, ny, nz = self.case.blocks[b].dims
        nf = {SETUP_METRICS: 9, SETUP_JACOBIAN: 1, SETUP_MEAN_GRADIENT: 5 * self.case.num_dim,
              SETUP_SPONGE: 1}[what]
        out = np.zeros((nf, nz, ny, nx))
        self._chk(self.lib.get_setup(self.ctx, b, what, _dptr(out)))
        return out


def _solver_info(self) -> LeeInfo:
    info = LeeInfo()
    self._chk(self.lib.get_info(self.ctx, C.byref(info)))
    return info


def _solver_stats(self) -> LeeStats:
    st = LeeStats()
    self._chk(self.lib.get_stats(self.ctx, C.byref(st)))
    return st


def _solver_timing(self, on: bool) -> None:
    self._chk(self.lib.set_timing(self.ctx, 1 if on else 0))


Solver.info = _solver_info
Solver.stats = _solver_stats
Solver.set_timing = _solver_timing


def _solver_graphs(self, on: bool) -> None:
    self._chk(self.lib.set_graphs(self.ctx, 1 if on else 0))


Solver.set_graphs = _solver_graphs


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 norm of a - b with respect to b."""
    nb = float(np.linalg.norm(b.ravel()))
    d = float(np.linalg.norm((a - b).ravel()))
    return d / nb if nb > 0 else d
