"""Synthetic LEE workloads: grids, mean flows, initial data and boundary lines.

Each builder returns a :class:`Case` that both the reference driver (through
PLOT3D files, a ``camille.in`` deck and a BC file) and this library's C ABI
consume, so every side starts from identical float64 arrays.

State and mean variables follow the reference's LEE layout
(src/core/param.h:67-80): slot 0 is entropy s', then u', v', w', p'.
The mean is (s_bar, u_bar, v_bar, w_bar, p_bar). An isentropic pulse has
s' = p'/(gamma p_bar) - rho'/rho_bar = 0 (src/core/state.cpp:701-736).

Workloads (sizes are parameters so tests can run them small):

* ``pulse2d``: 2-D Cartesian block on [-L/2, L/2]^2, quiescent mean
  (rho_bar = 1, u_bar = 0, p_bar = 1/gamma), Gaussian p' pulse of amplitude
  1e-3 and half-width 3 dx at the origin, ``exp(-ln2 r^2 / b^2)`` as in
  src/solver/source.cpp:69, Freund sponges ``width`` cells wide on all four
  sides (order 2, constant 5, as the example deck doc/inputDeck/examples/camille.in:35).
* ``curvi3d``: 3-D block with x = xi + 0.1 d sin(2 pi eta/L) sin(2 pi zeta/L)
  and its cyclic permutations (d = 1, L = n), uniform mean flow Mach 0.5 along
  x, eight Gaussian pulses (amplitude 1e-3, half-width 4 d) with centres drawn
  by ``numpy.random.default_rng(seed)``, no BC lines (boundary closures only).
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

from . import overset as overset_mod
from . import plot3d

BC_TYPES = {
    "dirichlet_allzero": 1,
    "dirichlet_harmonicwave": 2,
    "neumann": 100,
    "wall_slip_kinematic": 201,
    "centerline_cart_norm2x": 900,
    "centerline_cart_norm2y": 901,
    "centerline_cart_norm2z": 902,
    "centerline_axisym": 903,
    "sponge_freund_ambient": 1000,
    "sponge_freund_harmonicwave": 1002,
}
DIRS = {"XI": 0, "ETA": 1, "ZETA": 2}
WAVE_TYPES = {"WAVE_ACOUSTIC": 1, "WAVE_ENTROPY": 2}
WAVE_FORMS = {"WAVEFORM_PLANE": 0, "WAVEFORM_HOMOGENEOUS": 1, "WAVEFORM_GAUSSIAN_ROUNDJET": 2}


@dataclasses.dataclass
class Block:
    x: np.ndarray          # (nz, ny, nx) float64
    y: np.ndarray
    z: np.ndarray
    mean: np.ndarray       # (5, nz, ny, nx): s_bar, u_bar, v_bar, w_bar, p_bar
    state: np.ndarray      # (5, nz, ny, nx): s', u', v', w', p'
    iblank: Optional[np.ndarray] = None  # (nz, ny, nx) int32: 0 fluid, 1 hole, -1 receiver
    monopole: Optional[tuple[float, float, float, float, float, float, float]] = None  # this block's own
    zmean: Optional[np.ndarray] = None   # (n, nz, ny, nx): mean passive scalars Z_bar_k (LEE_SCALAR)
    zstate: Optional[np.ndarray] = None  # (n, nz, ny, nx): Z_k'

    @property
    def dims(self) -> tuple[int, int, int]:
        nz, ny, nx = self.x.shape
        return nx, ny, nz

    @property
    def npoints(self) -> int:
        return int(self.x.size)


@dataclasses.dataclass
class Boundary:
    """One BC-file line: ``iblock type +-dir is ie js je ks ke`` (inclusive, non-negative)."""
    block: int
    kind: str      # key of BC_TYPES
    dir: int       # 0 XI, 1 ETA, 2 ZETA
    end: int       # 0 left (+dir), 1 right (-dir)
    lo: tuple[int, int, int]
    hi: tuple[int, int, int]
    sigma: Optional[np.ndarray] = None  # sponge strengths over the box (i fastest), when precomputed

    def line(self) -> str:
        sign = "+" if self.end == 0 else "-"
        name = ["XI", "ETA", "ZETA"][self.dir]
        idx = []
        for d in range(3):
            idx += [str(self.lo[d]), str(self.hi[d])]
        return f"{self.block} {self.kind} {sign}{name} " + " ".join(idx)


@dataclasses.dataclass
class HarmonicWave:
    """The deck's ``HARMONIC_WAVE`` line (src/core/input.cpp:219-231), read by
    ``dirichlet_harmonicwave`` BC lines and ``sponge_freund_harmonicwave`` zones."""
    wave_type: str        # key of WAVE_TYPES
    form: str             # key of WAVE_FORMS
    direction: int        # 0 X, 1 Y, 2 Z
    amplitude: float
    wavelength: float
    halfwidth: float = 0.0  # WAVEFORM_GAUSSIAN_ROUNDJET only

    def args(self) -> tuple:
        """Arguments of lee_set_harmonic_wave after the context."""
        return (WAVE_TYPES[self.wave_type], WAVE_FORMS[self.form], self.direction, float(self.amplitude),
                float(self.wavelength), float(self.halfwidth))

    def deck_line(self) -> str:
        line = (f"HARMONIC_WAVE = {self.wave_type}, AMPLITUDE = {self.amplitude!r}, SHAPE = {self.form}, "
                f"DIRECTION = {'XYZ'[self.direction]}, WAVELENGTH = {self.wavelength!r}")
        if self.form == "WAVEFORM_GAUSSIAN_ROUNDJET":
            line += f", HALFWIDTH = {self.halfwidth!r}"
        return line


@dataclasses.dataclass
class DistributedSource:
    """rhs[p'] += (gamma - 1) sin(omega t) S on block ``block``, S the trilinear prolongation of
    ``amplitudes`` (shape (cz, cy, cx)) from lattice nodes at grid index origin + node * spacing
    (LEE_SOURCE_DISTRIBUTED of include/lee_b200.h; the reference has no such source)."""
    block: int
    omega: float
    origin: tuple[float, float, float]
    spacing: tuple[float, float, float]
    amplitudes: np.ndarray

    def params(self) -> np.ndarray:
        cz, cy, cx = self.amplitudes.shape
        head = [self.block, self.omega, cx, cy, cz, *self.origin, *self.spacing]
        return np.concatenate([np.asarray(head, np.float64), self.amplitudes.astype(np.float64).ravel()])


@dataclasses.dataclass
class Microphones:
    """Objective J = weight * sum over steps of sum over microphones of p'^2 at linear
    indices ``l0`` of block ``block``; weight None takes the FIX_CFL time step (a rectangle-rule
    time integral)."""
    block: int
    l0: np.ndarray
    weight: Optional[float] = None


# The pressure source of the reference's CASE_SCATTERING_TWOCYLINDER (src/solver/source.cpp:60-92),
# (gamma - 1) exp(-ln 2 r^2 / 0.2^2) sin(4 * 2 pi t) ramped by sin^2(pi/2 t / 4) up to t = 4, as
# monopole parameters (x0, y0, z0, amplitude, omega, halfwidth, ramp_time).
TWOCYLINDER_SOURCE = (0.0, 0.0, 0.0, 1.0, 4.0 * (2.0 * math.pi), 0.2, 16.0 / 4.0)


@dataclasses.dataclass
class Case:
    name: str
    num_dim: int
    blocks: list[Block]
    gamma: float = 1.4
    fd_scheme: str = "STANDARD_CENTRAL"    # or FDO11P
    fd_order: int = 4
    filter_scheme: str = "STANDARD_CENTRAL"  # STANDARD_CENTRAL, SFO11P or NONE
    filter_order: int = 8
    filter_strength: float = 1.0
    filter_blend: float = 1.0
    rk: str = "RUNGE_KUTTA4"
    cfl: float = 0.5
    nsteps: int = 1
    boundaries: list[Boundary] = dataclasses.field(default_factory=list)
    sponge_order: int = 2
    sponge_constant: float = 5.0
    monopole: Optional[tuple[float, float, float, float, float, float, float]] = None
    overset: Optional["overset_mod.OversetMap"] = None
    distributed: Optional[DistributedSource] = None
    microphones: Optional[Microphones] = None
    harmonic_wave: Optional[HarmonicWave] = None
    axisymmetric: bool = False  # AXISYMMETRY = TRUE, AXIS_OF_SYMMETRY = X (2-D: x axial, y radial)
    notes: str = ""
    # the deck's SIMULATION; CASE_SCATTERING_TWOCYLINDER brings the reference's own source
    simulation: str = "CASE_KBK_COMBUSTOR"

    @property
    def npoints(self) -> int:
        return sum(b.npoints for b in self.blocks)

    @property
    def num_scalars(self) -> int:
        """Passive scalars of PHYSICAL_MODEL = LEE_SCALAR (0: plain LEE)."""
        z = self.blocks[0].zmean
        return 0 if z is None else int(z.shape[0])

    def source_monopole(self) -> Optional[tuple[float, float, float, float, float, float, float]]:
        """The monopole that acts on every block: the case's own, else the one SIMULATION implies."""
        if self.monopole is not None:
            return self.monopole
        if self.simulation == "CASE_SCATTERING_TWOCYLINDER":
            return TWOCYLINDER_SOURCE
        return None

    # ---- reference input files -------------------------------------------------
    def deck_lines(self, dt: Optional[float], nsteps: int, grid: str, mean: str, bc: str,
                   report: int = 2000000000) -> list[str]:
        fix = "FIX_DT" if dt is not None else "FIX_CFL"
        lines = [
            f"DIMENSION = {self.num_dim}",
            "AXISYMMETRY = TRUE, AXIS_OF_SYMMETRY = X" if self.axisymmetric else "AXISYMMETRY = FALSE",
            (f"PHYSICAL_MODEL = LEE_SCALAR, NUMBER_SCALAR = {self.num_scalars}" if self.num_scalars
             else "PHYSICAL_MODEL = LEE"),
            "FLUID_MODEL = IDEAL_GAS_CALORIC",
            # the reference takes LEE_SCALAR only with CASE_LINEAR_NOZZLE (src/core/input.cpp:596-606);
            # its initial and mean states are replaced by the restart and base-state files
            f"SIMULATION = {'CASE_LINEAR_NOZZLE' if self.num_scalars else self.simulation}",
            f"GAMMA_SPECIFICHEAT = {self.gamma!r}",
            f"FIX_DT_OR_CFL = {fix}",
            f"DT = {dt!r}" if dt is not None else "DT = 1.0E-6",
            f"CFL = {self.cfl!r}",
            f"TEMPORAL_SCHEME = {self.rk}",
            f"NUM_TOTAL_TIMESTEP = {nsteps}",
            f"REPORT_TIMESTEP = {report}",
        ]
        if self.fd_scheme == "STANDARD_CENTRAL":
            lines.append(f"SPATIAL_SCHEME = STANDARD_CENTRAL, ORDER_ACCURACY = {self.fd_order}")
        else:
            lines.append(f"SPATIAL_SCHEME = {self.fd_scheme}")
        if self.filter_scheme == "STANDARD_CENTRAL":
            lines.append(f"SPATIAL_FILTER = STANDARD_CENTRAL, ORDER_ACCURACY = {self.filter_order}, "
                         f"BLEND = {self.filter_blend!r}")
        elif self.filter_scheme == "SFO11P":
            lines.append(f"SPATIAL_FILTER = SFO11P, STRENGTH = {self.filter_strength!r}, "
                         f"BLEND = {self.filter_blend!r}")
        else:
            lines.append("SPATIAL_FILTER = NONE")
        lines += [
            f"BUFFER_ZONE POLYNOMIAL_ORDER = {self.sponge_order}, CONSTANT = {self.sponge_constant!r}",
            "METRIC_SCHEME = THOMAS_LOMBARD",
        ]
        if self.overset is None:
            lines.append("OVERSET = NONE")
        else:
            lines.append(f"OVERSET = OVERTURE, TYPE = EXPLICIT, ORDER_ACCURACY = {self.overset.order}")
        lines += [
            "DOMAIN_DECOMPOSITION = DECOMP_1D",
            "FILE_FORMAT = PLOT3D",
            f"GRID_FILE = {grid}",
            f"BASESTATE_FILE = {mean}",
            f"BC_FILE = {bc}",
        ]
        if self.overset is not None:
            lines.append(f"OVERSET_FILE = {os.path.join(os.path.dirname(bc), 'overset.bin')}")
        lines += [
            "SOLUTION_WRITING_TIME = 1.0E+300",
            self.harmonic_wave.deck_line() if self.harmonic_wave is not None else "HARMONIC_WAVE = NONE",
            "INTERPOLATE_SOLUTION = NONE",
        ]
        if self.monopole is not None:
            # read by camille_b200/lee_run only; the reference never looks the name up
            lines.append("SOURCE_MONOPOLE = " + ", ".join(repr(float(v)) for v in self.monopole))
        return lines

    def write_reference_inputs(self, workdir: str, dt: Optional[float], nsteps: int,
                               step: int = 0, time: float = 0.0, report: int = 2000000000) -> str:
        """Write grid, mean, restart, BC and deck files; return the restart path."""
        if self.distributed is not None:
            raise ValueError("the reference cannot express a distributed source")
        if self.monopole is not None and self.simulation in ("CASE_SCATTERING_TWOCYLINDER",
                                                             "CASE_2DJET_WITH_A_HARMONIC_SOURCE"):
            raise ValueError("a case-level monopole and the case's own source do not combine")
        os.makedirs(workdir, exist_ok=True)
        grid, mean, ic, bc = (os.path.join(workdir, n) for n in ("grid.xyz", "mean.q", "ic.q", "bc.in"))
        plot3d.write_grid(grid, [(b.x, b.y, b.z) for b in self.blocks])
        if self.num_scalars:
            plot3d.write_function(mean, [np.concatenate([b.mean, b.zmean]) for b in self.blocks])
            plot3d.write_solution(ic, [np.concatenate([b.state, b.zstate]) for b in self.blocks], step=step,
                                  time=time)
        else:
            plot3d.write_function(mean, [b.mean for b in self.blocks])
            plot3d.write_solution(ic, [b.state for b in self.blocks], step=step, time=time)
        plot3d.write_bc(bc, [bd.line() for bd in self.boundaries])
        if self.overset is not None:
            self.overset.write(os.path.join(workdir, "overset.bin"))
        plot3d.write_deck(os.path.join(workdir, "camille.in"), self.deck_lines(dt, nsteps, grid, mean, bc, report))
        return ic


def _gauss(r2: np.ndarray, halfwidth: float) -> np.ndarray:
    return np.exp(-math.log(2.0) * r2 / (halfwidth * halfwidth))


def sponge_frame(num_dim: int, dims: tuple[int, int, int], width: int, block: int = 0) -> list[Boundary]:
    """Freund ambient sponges ``width`` cells wide on every side of a block."""
    out = []
    nmax = [d - 1 for d in dims]
    for d in range(num_dim):
        for end in (0, 1):
            lo = [0, 0, 0]
            hi = list(nmax)
            if end == 0:
                hi[d] = width - 1
            else:
                lo[d] = nmax[d] - (width - 1)
            out.append(Boundary(block, "sponge_freund_ambient", d, end, tuple(lo), tuple(hi)))
    return out


def pulse2d(n: int = 256, length: float = 100.0, sponge: int = 20, nsteps: int = 1000,
            gamma: float = 1.4) -> Case:
    dx = length / (n - 1)
    c1 = -0.5 * length + dx * np.arange(n, dtype=np.float64)
    y, x = np.meshgrid(c1, c1, indexing="ij")
    x = x[None].copy()
    y = y[None].copy()
    z = np.zeros_like(x)
    mean = np.zeros((5,) + x.shape)
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    state[4] = 1e-3 * _gauss(x * x + y * y, 3.0 * dx)
    blk = Block(x, y, z, mean, state)
    bnd = sponge_frame(2, blk.dims, sponge) if sponge > 0 else []
    return Case(name=f"pulse2d_{n}", num_dim=2, blocks=[blk], gamma=gamma, nsteps=nsteps,
                boundaries=bnd,
                notes=f"2-D {n}^2 on [-{length/2},{length/2}]^2, quiescent, sponge {sponge}")


def curvi3d_grid(n: int, amp: float = 0.1) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    L = float(n)
    c = np.arange(n, dtype=np.float64)
    zeta, eta, xi = np.meshgrid(c, c, c, indexing="ij")
    s = lambda a: np.sin(2.0 * math.pi * a / L)  # noqa: E731
    x = xi + amp * s(eta) * s(zeta)
    y = eta + amp * s(zeta) * s(xi)
    z = zeta + amp * s(xi) * s(eta)
    return x, y, z


def curvi3d(n: int = 256, seed: int = 2, npulses: int = 8, mach: float = 0.5, nsteps: int = 500,
            gamma: float = 1.4, halfwidth: float = 4.0, sponge: int = 0, sponge_constant: float = 1.0) -> Case:
    x, y, z = curvi3d_grid(n)
    mean = np.zeros((5,) + x.shape)
    mean[1] = mach
    mean[4] = 1.0 / gamma
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2 * (n - 1), 0.8 * (n - 1), size=(npulses, 3))
    p = np.zeros(x.shape)
    for cx, cy, cz in centres:
        p += 1e-3 * _gauss((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2, halfwidth)
    state = np.zeros((5,) + x.shape)
    state[4] = p
    blk = Block(x, y, z, mean, state)
    bnd = sponge_frame(3, blk.dims, sponge) if sponge > 0 else []
    return Case(name=f"curvi3d_{n}", num_dim=3, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=sponge_constant,
                notes=f"3-D {n}^3 curvilinear, Mach {mach} along x, {npulses} pulses seed {seed}, "
                      f"sponge {sponge} (constant {sponge_constant})")


def sponge_sigma(case: Case, bd: Boundary) -> np.ndarray:
    """Freund sponge strengths of one zone, C (d_in / (d_in + d_out))^order, where d_in/d_out are
    the distances to the nearest grid point of the zone's inner/outer face
    (Geometry::additionalInit_bufferZones, src/geometry/geometry.cpp:1028-1142). The reference
    searches every face point for every zone point; an exact nearest-neighbour search over the
    same points gives the same minimum distance in O(N log N)."""
    from scipy.spatial import cKDTree

    blk = case.blocks[bd.block]
    xyz = np.stack([blk.x, blk.y, blk.z], axis=-1)  # (nz, ny, nx, 3)
    sl = tuple(slice(bd.lo[d], bd.hi[d] + 1) for d in (2, 1, 0))
    pts = xyz[sl].reshape(-1, 3)
    ax = 2 - bd.dir  # numpy axis of the zone's direction

    def face(index: int) -> np.ndarray:
        f = list(sl)
        f[ax] = slice(index, index + 1)
        return xyz[tuple(f)].reshape(-1, 3)

    f_in = face(bd.hi[bd.dir] if bd.end == 0 else bd.lo[bd.dir])
    f_out = face(bd.lo[bd.dir] if bd.end == 0 else bd.hi[bd.dir])
    d_in = cKDTree(f_in).query(pts)[0]
    d_out = cKDTree(f_out).query(pts)[0]
    rel = d_in / (d_in + d_out)
    return (case.sponge_constant * rel ** case.sponge_order).astype(np.float64)


def precompute_sponges(case: Case) -> None:
    """Fill Boundary.sigma for every sponge of the case (used for large blocks)."""
    for bd in case.boundaries:
        if bd.kind == "sponge_freund_ambient" and bd.sigma is None:
            bd.sigma = sponge_sigma(case, bd)


def shear2d(nx: int = 64, ny: int = 48, spacing: float = 0.25, bump: float = 0.3, nsteps: int = 10,
            sponge: int = 6, gamma: float = 1.4, halfwidth: float = 4.0) -> Case:
    """2-D block over a bumped slip wall under a parallel tanh shear layer.

    The wall (eta = 0) follows y_w(x) = bump * exp(-x^2 / (ny spacing)^2 * 16) and the grid
    lines relax to flat at the top; the mean is u_bar = 0.15 (1 + tanh 2 (y - y_c)) with
    y_c at mid height, a mild entropy layer s_bar = 0.05 tanh(y - y_c) and p_bar = 1/gamma,
    so every mean-gradient term of the right-hand side, including the rho'/rho_bar one, is
    active. BC lines: ``wall_slip_kinematic`` on the wall, ``neumann`` on the top, Freund
    sponges ``sponge`` cells wide at both x ends. A Gaussian p' pulse sits over the bump and a
    weaker one below the top face."""
    xs = (np.arange(nx, dtype=np.float64) - 0.5 * (nx - 1)) * spacing
    eta = np.arange(ny, dtype=np.float64)
    height = (ny - 1) * spacing
    yw = bump * np.exp(-16.0 * xs * xs / (height * height))
    frac = eta / (ny - 1)
    x = np.broadcast_to(xs[None, :], (ny, nx)).copy()
    y = yw[None, :] * (1.0 - frac[:, None]) + (eta * spacing)[:, None]
    x, y = x[None], y[None]
    z = np.zeros_like(x)
    yc = 0.5 * height
    mean = np.zeros((5,) + x.shape)
    mean[0] = 0.05 * np.tanh(y - yc)
    mean[1] = 0.15 * (1.0 + np.tanh(2.0 * (y - yc)))
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    state[4] = 1e-3 * _gauss(x * x + (y - 0.3 * height) ** 2, halfwidth * spacing)
    state[4] += 5e-4 * _gauss((x - 0.2 * xs[-1]) ** 2 + (y - 0.85 * height) ** 2, halfwidth * spacing)
    blk = Block(x, y, z, mean, state)
    bnd = [Boundary(0, "wall_slip_kinematic", 1, 0, (0, 0, 0), (nx - 1, 0, 0)),
           Boundary(0, "neumann", 1, 1, (0, ny - 1, 0), (nx - 1, ny - 1, 0))]
    if sponge > 0:
        bnd += [b for b in sponge_frame(2, blk.dims, sponge) if b.dir == 0]
    return Case(name=f"shear2d_{nx}x{ny}", num_dim=2, blocks=[blk], gamma=gamma, nsteps=nsteps,
                boundaries=bnd, sponge_constant=1.0,
                notes=f"2-D {nx}x{ny} shear layer over a bumped slip wall, sponge {sponge}")


def wall3d(n: int = 16, nsteps: int = 3, gamma: float = 1.4, halfwidth: float = 2.0) -> Case:
    """3-D curvilinear block (the curvi3d mapping) with a slip wall on zeta = 0, a Neumann
    face on xi = n-1 and a mean shear u_bar = 0.3 (1 + 0.5 tanh((z - n/2) / 3)) along x,
    so that the rho'/rho_bar term is active in 3-D too."""
    x, y, z = curvi3d_grid(n)
    mean = np.zeros((5,) + x.shape)
    mean[1] = 0.3 * (1.0 + 0.5 * np.tanh((z - 0.5 * n) / 3.0))
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    c = 0.5 * (n - 1)
    state[4] = 1e-3 * _gauss((x - c) ** 2 + (y - c) ** 2 + (z - 0.3 * n) ** 2, halfwidth)
    blk = Block(x, y, z, mean, state)
    m = n - 1
    bnd = [Boundary(0, "wall_slip_kinematic", 2, 0, (0, 0, 0), (m, m, 0)),
           Boundary(0, "neumann", 0, 1, (m, 0, 0), (m, m, m))]
    return Case(name=f"wall3d_{n}", num_dim=3, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                notes=f"3-D {n}^3 curvilinear, slip wall zeta=0, Neumann xi=max, shear mean")


def waves2d(nx: int = 40, ny: int = 32, spacing: float = 0.25, nsteps: int = 10, gamma: float = 1.4,
            wave: Optional[HarmonicWave] = None, mach: float = 0.2, sponge: int = 8) -> Case:
    """2-D Cartesian block on [0, (nx-1) d] x [0, (ny-1) d] driven by a time-harmonic wave
    (by default an acoustic plane wave along x, amplitude 1e-3, wavelength 16 d) under a
    uniform mean flow of Mach ``mach`` along x. BC lines: ``dirichlet_harmonicwave`` on xi = 0,
    ``centerline_cart_norm2y`` on eta = 0, ``dirichlet_allzero`` on eta = max, ``neumann`` on
    xi = max, and a ``sponge_freund_harmonicwave`` zone ``sponge`` cells wide at the xi = max
    end that relaxes toward the same wave. A weak Gaussian p' pulse starts inside."""
    if wave is None:
        wave = HarmonicWave("WAVE_ACOUSTIC", "WAVEFORM_PLANE", 0, 1e-3, 16.0 * spacing)
    xs = np.arange(nx, dtype=np.float64) * spacing
    ys = np.arange(ny, dtype=np.float64) * spacing
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    z = np.zeros_like(x)
    mean = np.zeros((5,) + x.shape)
    mean[1] = mach
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    state[4] = 5e-4 * _gauss((x - 0.5 * xs[-1]) ** 2 + (y - 0.4 * ys[-1]) ** 2, 3.0 * spacing)
    blk = Block(x, y, z, mean, state)
    mx, my = nx - 1, ny - 1
    bnd = [Boundary(0, "dirichlet_harmonicwave", 0, 0, (0, 0, 0), (0, my, 0)),
           Boundary(0, "centerline_cart_norm2y", 1, 0, (0, 0, 0), (mx, 0, 0)),
           Boundary(0, "dirichlet_allzero", 1, 1, (0, my, 0), (mx, my, 0)),
           Boundary(0, "neumann", 0, 1, (mx, 0, 0), (mx, my, 0))]
    if sponge > 0:
        bnd.append(Boundary(0, "sponge_freund_harmonicwave", 0, 1, (mx - sponge + 1, 0, 0), (mx, my, 0)))
    return Case(name=f"waves2d_{nx}x{ny}", num_dim=2, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=2.0, harmonic_wave=wave,
                notes=f"2-D {nx}x{ny} harmonic wave {wave.wave_type}/{wave.form}, centerline, allzero, sponge")


def jet3d(n: int = 14, nsteps: int = 4, gamma: float = 1.4, wave: Optional[HarmonicWave] = None,
          mach: float = 0.3, sponge: int = 4) -> Case:
    """3-D curvilinear block (the curvi3d mapping) with the corner eta = zeta = 0 as the axis of
    a quarter round jet: an entropy wave (by default the Gaussian round jet along x, amplitude
    1e-3, wavelength 6, half-width 3) enters through a ``dirichlet_harmonicwave`` face on
    xi = 0 and a ``sponge_freund_harmonicwave`` zone ``sponge`` cells deep behind it, under a
    uniform mean flow of Mach ``mach`` along x; ``centerline_cart_norm2y`` on eta = 0,
    ``centerline_cart_norm2z`` on zeta = 0, ``neumann`` on eta = max and zeta = max, and an
    ambient sponge at the xi = max end."""
    if wave is None:
        wave = HarmonicWave("WAVE_ENTROPY", "WAVEFORM_GAUSSIAN_ROUNDJET", 0, 1e-3, 6.0, 3.0)
    x, y, z = curvi3d_grid(n)
    mean = np.zeros((5,) + x.shape)
    mean[1] = mach
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    c = 0.5 * (n - 1)
    state[4] = 5e-4 * _gauss((x - c) ** 2 + (y - 0.3 * n) ** 2 + (z - 0.3 * n) ** 2, 2.0)
    blk = Block(x, y, z, mean, state)
    m = n - 1
    bnd = [Boundary(0, "dirichlet_harmonicwave", 0, 0, (0, 0, 0), (0, m, m)),
           Boundary(0, "centerline_cart_norm2y", 1, 0, (0, 0, 0), (m, 0, m)),
           Boundary(0, "centerline_cart_norm2z", 2, 0, (0, 0, 0), (m, m, 0)),
           Boundary(0, "neumann", 1, 1, (0, m, 0), (m, m, m)),
           Boundary(0, "neumann", 2, 1, (0, 0, m), (m, m, m))]
    if sponge > 0:
        bnd += [Boundary(0, "sponge_freund_harmonicwave", 0, 0, (0, 0, 0), (sponge - 1, m, m)),
                Boundary(0, "sponge_freund_ambient", 0, 1, (m - sponge + 1, 0, 0), (m, m, m))]
    return Case(name=f"jet3d_{n}", num_dim=3, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=1.0, harmonic_wave=wave,
                notes=f"3-D {n}^3 quarter jet, harmonic wave {wave.wave_type}/{wave.form}, centerlines")


def axisym2d(nx: int = 48, nr: int = 32, spacing: float = 0.125, nsteps: int = 10, gamma: float = 1.4,
             mach: float = 0.3, sponge: int = 6, halfwidth: float = 3.0) -> Case:
    """Axisymmetric round jet in the (x, r) half-plane (AXISYMMETRY = TRUE, axis x): x on
    [-(nx-1) d / 2, (nx-1) d / 2], r = y on [0, (nr-1) d] with the axis as the eta = 0 line;
    mean u_bar = mach (1 - tanh((r - 1) / 0.25)) / 2 and an entropy layer of the same shape
    (s_bar = 0.05 times it), v_bar = 0, p_bar = 1/gamma. BC lines: ``centerline_axisym`` on the
    axis, ``neumann`` on eta = max, Freund sponges ``sponge`` cells wide at both x ends. A
    Gaussian p' pulse sits on the axis."""
    xs = (np.arange(nx, dtype=np.float64) - 0.5 * (nx - 1)) * spacing
    rs = np.arange(nr, dtype=np.float64) * spacing
    x = np.broadcast_to(xs[None, None, :], (1, nr, nx)).copy()
    y = np.broadcast_to(rs[None, :, None], (1, nr, nx)).copy()
    z = np.zeros_like(x)
    prof = 0.5 * (1.0 - np.tanh((y - 1.0) / 0.25))
    mean = np.zeros((5,) + x.shape)
    mean[0] = 0.05 * prof
    mean[1] = mach * prof
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + x.shape)
    state[4] = 1e-3 * _gauss((x + 0.1 * xs[-1]) ** 2 + y * y, halfwidth * spacing)
    blk = Block(x, y, z, mean, state)
    mx, my = nx - 1, nr - 1
    bnd = [Boundary(0, "centerline_axisym", 1, 0, (0, 0, 0), (mx, 0, 0)),
           Boundary(0, "neumann", 1, 1, (0, my, 0), (mx, my, 0))]
    if sponge > 0:
        bnd += [b for b in sponge_frame(2, blk.dims, sponge) if b.dir == 0]
    return Case(name=f"axisym2d_{nx}x{nr}", num_dim=2, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=1.0, axisymmetric=True,
                notes=f"2-D axisymmetric round jet {nx}x{nr}, axis centerline, sponges at both x ends")


def jet2d_source(nx: int = 64, ny: int = 48, spacing: float = 0.25, nsteps: int = 10, gamma: float = 1.4,
                 sponge: int = 8) -> Case:
    """SIMULATION = CASE_2DJET_WITH_A_HARMONIC_SOURCE: the reference's own harmonic pressure
    source (src/solver/source.cpp:27-58) in its parallel hot jet, on a Cartesian block centred on
    the source with Freund sponges on all four sides. The mean is the one the reference's
    initializer gives (State::initialize_state_linearizedEuler_2Djet_with_a_harmonic_source,
    src/core/state.cpp:376-464: T_j = 600 K over 300 K ambient, M_j = 0.756, u_bar = u_j
    exp(-ln 2 y^2), the Crocco-Busemann density of its eq. (19)); the state starts at zero."""
    xs = (np.arange(nx, dtype=np.float64) - 0.5 * (nx - 1)) * spacing
    ys = (np.arange(ny, dtype=np.float64) - 0.5 * (ny - 1)) * spacing
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    z = np.zeros_like(x)
    pbar = 1.0 / gamma
    tj = 600.0 / ((gamma - 1.0) * 300.0)
    cj = math.sqrt((gamma - 1.0) * tj)
    uj = 0.756 * cj
    rhoj = pbar * gamma / (gamma - 1.0) / tj
    ubar = uj * np.exp(-math.log(2.0) * y ** 2)
    rhobar = 1.0 / (-0.5 * (gamma - 1.0) * (ubar - uj) * ubar + ubar / (rhoj * uj) + (uj - ubar) / uj)
    mean = np.zeros((5,) + x.shape)
    mean[0] = (0.0 - gamma * np.log(rhobar)) / gamma
    mean[1] = ubar
    mean[4] = pbar
    state = np.zeros((5,) + x.shape)
    blk = Block(x, y, z, mean, state)
    bnd = sponge_frame(2, blk.dims, sponge) if sponge > 0 else []
    return Case(name=f"jet2d_source_{nx}x{ny}", num_dim=2, blocks=[blk], gamma=gamma, nsteps=nsteps,
                boundaries=bnd, sponge_constant=1.0, simulation="CASE_2DJET_WITH_A_HARMONIC_SOURCE",
                notes=f"2-D {nx}x{ny} hot jet with the reference's harmonic pressure source")


def _tanh_radii(nr: int, r0: float, r1: float, first: float) -> tuple[np.ndarray, float]:
    """r(s) = r0 + (r1 - r0) (1 + tanh(d (s - 1)) / tanh d), s = j / (nr - 1), with d chosen so
    that the first cell is ``first`` wide (one-sided tanh clustering at the wall)."""
    from scipy.optimize import brentq

    def first_cell(d: float) -> float:
        return (r1 - r0) * (1.0 + math.tanh(d * (1.0 / (nr - 1) - 1.0)) / math.tanh(d)) - first

    d = brentq(first_cell, 1e-6, 50.0, xtol=1e-15, rtol=1e-15)
    s = np.arange(nr, dtype=np.float64) / (nr - 1)
    return r0 + (r1 - r0) * (1.0 + np.tanh(d * (s - 1.0)) / math.tanh(d)), d


def cylinder2d(nb: int = 512, length: float = 80.0, ntheta: int = 384, nr: int = 96, r_wall: float = 0.5,
               r_out: float = 5.0, first_cell: float = 0.005, r_cut: float = 1.5, seam_overlap: float = 8.5,
               fringe: int = 2, sponge: Optional[int] = None, sponge_constant: float = 5.0,
               source: tuple[float, float] = (2.0, 0.0), omega: float = 0.8 * math.pi, halfwidth: float = 0.2,
               amplitude: float = 1e-3, ramp: float = 2.5, nsteps: int = 4000, gamma: float = 1.4,
               pulse: Optional[tuple[float, float, float, float]] = None, wall_damping: float = 0.5) -> Case:
    """Two-block overset workload: a Cartesian background (block 0, nb x nb on [-L/2, L/2]^2)
    and a body-fitted O-grid (block 1, ntheta x nr) around a cylinder of radius ``r_wall``,
    radii clustered at the wall by a one-sided tanh (first cell ``first_cell``) out to ``r_out``.

    The reference has no periodic boundary, so the O-grid wraps past 2 pi by ``seam_overlap``
    cells: its first and last ``fringe`` theta lines are receivers donated by the O-grid's
    own interior across the seam. The background is blanked inside ``r_cut`` and its
    ``fringe`` layers of points next to the hole are receivers donated by the O-grid; the
    O-grid's outer ``fringe`` rings are receivers donated by the background. Donor stencils
    are 4 x 4 Lagrange (``ORDER_ACCURACY = 3``) in the donor's computational coordinates.

    Mean flow: the parallel shear layer u_bar = 0.15 (1 + tanh 2y) (Mach units, c = 1:
    rho_bar = 1, p_bar = 1/gamma) on both blocks, times 1 - exp(-((r - r_wall) / wall_damping)^2)
    so that it vanishes at the cylinder. A parallel mean taken straight through the body
    enters the domain through the wall behind the cylinder, where a slip wall cannot be a
    well-posed boundary; in the reference's arithmetic that run grows without bound after
    about 1400 steps at the full size. ``wall_damping = 0`` keeps the undamped layer. Source: monopole at ``source`` with
    angular frequency ``omega``, Gaussian half-width ``halfwidth`` and a sin^2 ramp over
    ``ramp``. BC lines: slip wall on the cylinder (O-grid eta = 0) and Freund sponges on the
    background's four sides (``sponge`` cells, default 20 at nb = 512). The initial state is
    zero, or a Gaussian p' pulse ``pulse`` = (x0, y0, amplitude, half-width) on both blocks."""
    # background
    dx = length / (nb - 1)
    c1 = -0.5 * length + dx * np.arange(nb, dtype=np.float64)
    yb, xb = np.meshgrid(c1, c1, indexing="ij")
    # O-grid: theta decreases with i so that the mapping is right-handed (positive Jacobian)
    period = ntheta - 1 - seam_overlap
    dth = 2.0 * math.pi / period
    radii, delta = _tanh_radii(nr, r_wall, r_out, first_cell)
    th = -dth * np.arange(ntheta, dtype=np.float64)
    xo = radii[:, None] * np.cos(th)[None, :]
    yo = radii[:, None] * np.sin(th)[None, :]

    def block(x2: np.ndarray, y2: np.ndarray) -> Block:
        x, y = x2[None].copy(), y2[None].copy()
        mean = np.zeros((5,) + x.shape)
        mean[1] = 0.15 * (1.0 + np.tanh(2.0 * y))
        if wall_damping > 0.0:
            rr = np.hypot(x, y)
            mean[1] *= 1.0 - np.exp(-(np.maximum(rr - r_wall, 0.0) / wall_damping) ** 2)
        mean[4] = 1.0 / gamma
        return Block(x, y, np.zeros_like(x), mean, np.zeros((5,) + x.shape))

    bg, og = block(xb, yb), block(xo, yo)
    if pulse is not None:
        px, py, pa, pb = pulse
        for blk in (bg, og):
            blk.state[4] = pa * _gauss((blk.x - px) ** 2 + (blk.y - py) ** 2, pb)

    # background hole and fringe
    ib_bg = np.zeros((nb, nb), np.int32)
    hole = np.hypot(xb, yb) < r_cut
    ib_bg[hole] = overset_mod.BLANKED
    near = np.zeros_like(hole)
    hj, hi = np.nonzero(hole)
    for dj in range(-fringe, fringe + 1):
        for di in range(-fringe, fringe + 1):
            jj, ii = np.clip(hj + dj, 0, nb - 1), np.clip(hi + di, 0, nb - 1)
            near[jj, ii] = True
    recv_bg = near & ~hole
    ib_bg[recv_bg] = overset_mod.INTERPOLATED
    # O-grid receivers: outer rings, then the seam lines
    recv_og = np.zeros((nr, ntheta), bool)
    recv_og[nr - fringe:, :] = True
    seam = np.zeros_like(recv_og)
    seam[:nr - fringe, :fringe] = True
    seam[:nr - fringe, ntheta - fringe:] = True
    recv_og |= seam

    def inv_bg(x: float, y: float):
        return [((x + 0.5 * length) / dx, (y + 0.5 * length) / dx)]

    tanh_d = math.tanh(delta)

    def inv_og(x: float, y: float):
        r = math.hypot(x, y)
        t = ((r - r_wall) / (r_out - r_wall) - 1.0) * tanh_d
        if not (-1.0 < t <= 0.0):
            return []
        eta = (nr - 1) * (1.0 + math.atanh(t) / delta)
        xi = ((-math.atan2(y, x)) % (2.0 * math.pi)) / dth
        return [(xi, eta), (xi + period, eta), (xi - period, eta)]

    donors = [overset_mod.DonorGrid((nb, nb), inv_bg, ib_bg == overset_mod.NOTBLANKED),
              overset_mod.DonorGrid((ntheta, nr), inv_og, ~recv_og)]
    rb, rijk, db, dijk, wts = [], [], [], [], []

    def add(block_id: int, mask: np.ndarray, xs: np.ndarray, ys: np.ndarray, donor_of) -> None:
        jj, ii = np.nonzero(mask)
        order = np.lexsort((ii, jj))  # i fastest
        for q in order:
            j, i = int(jj[q]), int(ii[q])
            d = donor_of(i, j)
            found = overset_mod.find_donor(donors[d], float(xs[j, i]), float(ys[j, i]))
            if found is None:
                raise ValueError(f"no donor stencil for block {block_id} point ({i}, {j}) in block {d}")
            i0, j0, w = found
            rb.append(block_id); rijk.append((i, j, 0)); db.append(d); dijk.append((i0, j0, 0)); wts.append(w)

    add(0, recv_bg, xb, yb, lambda i, j: 1)
    add(1, recv_og, xo, yo, lambda i, j: 0 if j >= nr - fringe else 1)
    hj, hi = np.nonzero(hole)
    order = np.lexsort((hi, hj))
    ovs = overset_mod.OversetMap(
        num_dim=2, block_points=[nb * nb, ntheta * nr],
        recv_block=np.asarray(rb, np.int32), recv_ijk=np.asarray(rijk, np.int32),
        donor_block=np.asarray(db, np.int32), donor_ijk=np.asarray(dijk, np.int32), width=(4, 4, 1),
        weights=np.asarray(wts, np.float64), hole_block=np.zeros(order.size, np.int32),
        hole_ijk=np.stack([hi[order], hj[order], np.zeros(order.size, np.int64)], axis=1).astype(np.int32))
    if sponge is None:
        sponge = max(4, int(round(20 * nb / 512)))
    bnd = [Boundary(1, "wall_slip_kinematic", 1, 0, (0, 0, 0), (ntheta - 1, 0, 0))]
    bnd += sponge_frame(2, bg.dims, sponge, block=0) if sponge > 0 else []
    return Case(name=f"cylinder2d_{nb}_{ntheta}x{nr}", num_dim=2, blocks=[bg, og], gamma=gamma, nsteps=nsteps,
                boundaries=bnd, sponge_constant=sponge_constant, overset=ovs,
                monopole=(source[0], source[1], 0.0, amplitude, omega, halfwidth, ramp),
                notes=f"2-D overset: background {nb}^2 on [-{length/2},{length/2}]^2, O-grid {ntheta}x{nr} "
                      f"r in [{r_wall},{r_out}] first cell {first_cell}, shear layer, monopole at {source}")


def adjoint3d(n: int = 192, nsteps: int = 2000, seed: int = 5, mach: float = 0.5, lattice: int = 16,
              omega: float = 0.4 * math.pi, amp_std: float = 1e-3, nmics: int = 64, gamma: float = 1.4,
              sponge: Optional[int] = None, precompute: bool = False) -> Case:
    """The adjoint workload: the curvi3d mapping at n^3, Mach ``mach`` along x, zero initial
    state, a distributed monopole whose lattice x lattice x lattice amplitudes are drawn
    N(0, amp_std) from ``numpy.random.default_rng(seed)`` and span 60 n/192 grid cells around
    the block centre (node spacing 4 n/192), at angular frequency ``omega``; ``nmics``
    microphones on the downstream half circle of radius 60 n/192 cells in the mid-zeta plane;
    Freund sponges n/16 cells wide (constant 1), as the 256^3 workload."""
    x, y, z = curvi3d_grid(n)
    mean = np.zeros((5,) + x.shape)
    mean[1] = mach
    mean[4] = 1.0 / gamma
    blk = Block(x, y, z, mean, np.zeros((5,) + x.shape))
    width = max(4, int(round(n / 16))) if sponge is None else sponge
    bnd = sponge_frame(3, blk.dims, width) if width > 0 else []
    c = 0.5 * (n - 1)
    h = 4.0 * n / 192.0
    o = c - 0.5 * (lattice - 1) * h
    rng = np.random.default_rng(seed)
    amps = rng.normal(0.0, amp_std, size=(lattice, lattice, lattice))
    src = DistributedSource(0, omega, (o, o, o), (h, h, h), amps)
    R = 60.0 * n / 192.0
    th = np.linspace(-0.5 * math.pi, 0.5 * math.pi, nmics)
    ii = np.rint(c + R * np.cos(th)).astype(np.int64)
    jj = np.rint(c + R * np.sin(th)).astype(np.int64)
    kk = n // 2
    l0 = ii + n * (jj + n * kk)
    if np.unique(l0).size != l0.size:
        raise ValueError("microphones collide at this size")
    case = Case(name=f"adjoint3d_{n}", num_dim=3, blocks=[blk], gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=1.0, distributed=src, microphones=Microphones(0, l0),
                notes=f"3-D {n}^3 curvilinear, Mach {mach}, distributed source {lattice}^3 (seed {seed}), "
                      f"{nmics} microphones r = {R:.1f}")
    if precompute:
        precompute_sponges(case)
    return case


def batch2d(count: int = 64, seed: int = 4, nmin: int = 64, nmax: int = 512, nsteps: int = 2000,
            spacing: float = 100.0 / 255.0, gamma: float = 1.4, sponge_constant: float = 5.0,
            spacing_spread: float = 1.0) -> Case:
    """A batch of ``count`` independent square 2-D Cartesian instances (one block each) drawn by
    ``numpy.random.default_rng(seed)``: side N = round(exp(U[ln nmin, ln nmax])) points at
    ``spacing``, uniform mean Mach U[0, 0.6] along x, a monopole at a uniform position inside the
    central half of the instance with angular frequency U[pi/10, pi/3], amplitude 1e-3, Gaussian
    half-width 3 spacings and a sin^2 ramp over one period, and Freund sponges 20 N/256 cells
    wide (at least 4) on every side. Each instance advances with its own CFL time step.
    ``spacing_spread`` > 1 draws each instance's spacing log-uniformly in
    [spacing / spread, spacing * spread] (after the draws above, so they are unchanged)."""
    rng = np.random.default_rng(seed)
    sides = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count))).astype(int)
    draws = [(float(rng.uniform(0.0, 0.6)), float(rng.uniform(math.pi / 10.0, math.pi / 3.0)),
              rng.uniform(-0.25, 0.25, size=2)) for _ in range(count)]
    spacings = [spacing] * count
    if spacing_spread > 1.0:
        spacings = list(spacing * np.exp(rng.uniform(-math.log(spacing_spread), math.log(spacing_spread), count)))
    blocks, bnd = [], []
    for b, n in enumerate(sides):
        n = int(n)
        spacing = float(spacings[b])
        mach, omega, pos = draws[b]
        length = (n - 1) * spacing
        sx, sy = pos * length
        c1 = -0.5 * length + spacing * np.arange(n, dtype=np.float64)
        y, x = np.meshgrid(c1, c1, indexing="ij")
        x, y = x[None].copy(), y[None].copy()
        mean = np.zeros((5,) + x.shape)
        mean[1] = mach
        mean[4] = 1.0 / gamma
        blk = Block(x, y, np.zeros_like(x), mean, np.zeros((5,) + x.shape),
                    monopole=(float(sx), float(sy), 0.0, 1e-3, omega, 3.0 * spacing, 2.0 * math.pi / omega))
        blocks.append(blk)
        width = max(4, int(round(20 * n / 256)))
        bnd += sponge_frame(2, blk.dims, width, block=b)
    return Case(name=f"batch2d_{count}", num_dim=2, blocks=blocks, gamma=gamma, nsteps=nsteps, boundaries=bnd,
                sponge_constant=sponge_constant,
                notes=f"{count} 2-D instances, sides {int(sides.min())}..{int(sides.max())}, seed {seed}")


def instance(case: Case, b: int) -> Case:
    """Block b of a batch as a single-block case of its own (its boundaries renumbered)."""
    blk = case.blocks[b]
    bnd = [dataclasses.replace(bd, block=0) for bd in case.boundaries if bd.block == b]
    return dataclasses.replace(case, name=f"{case.name}_b{b}", blocks=[blk], boundaries=bnd)


def _boxes_mask(dims: tuple[int, int, int], boxes) -> np.ndarray:
    """(nz, ny, nx) bool mask of the union of inclusive index boxes ((i0, i1), (j0, j1), (k0, k1))."""
    nx, ny, nz = dims
    m = np.zeros((nz, ny, nx), bool)
    for (i0, i1), (j0, j1), (k0, k1) in boxes:
        m[k0:k1 + 1, j0:j1 + 1, i0:i1 + 1] = True
    return m


def holes(num_dim: int = 2, nsteps: int = 12, seed: int = 11, gamma: float = 1.4) -> Case:
    """A single Cartesian block (64 x 56 in 2-D, 24^3 in 3-D, unit spacing) with a hand-set pattern of
    holes and receivers, so that every branch of the reference's hole closures
    (StandardCentral::iblank_correction, src/solver/spatial_discretization.cpp:1356-1652) occurs
    along every direction: a hole after a plain fluid point (the ``last_iblank /= BLANKED``
    branch that inserts no closure), a hole after a receiver (right closure rows anchored at
    the receiver), a hole after a hole (zero), fluid and receivers after a hole (left closure
    rows), holes at the start and at the end of lines, and a seven-point run between a hole at a
    line start and a hole after receivers (the filter closure's whole support).

    Receivers are donated by the block itself (4-point stencils in every direction, positive
    seeded weights) from a fluid region away from holes and receivers. Uniform mean flow
    (Mach 0.3, 0.2, 0.1 along x, y, z), a Gaussian p' pulse over the holes, closures at the block
    edges and no BC lines. The maps go to both sides through the reference's overset file."""
    rng = np.random.default_rng(seed)
    if num_dim == 2:
        dims = (64, 56, 1)
        z1 = (0, 0)
        hole_boxes = [((20, 24), (10, 14), z1), ((40, 44), (10, 14), z1), ((0, 3), (26, 30), z1),
                      ((58, 63), (26, 30), z1), ((20, 26), (52, 55), z1), ((40, 46), (0, 2), z1)]
        recv_boxes = [((38, 39), (10, 14), z1), ((45, 46), (10, 14), z1), ((40, 44), (8, 9), z1),
                      ((40, 44), (15, 16), z1), ((56, 57), (26, 30), z1), ((20, 26), (50, 51), z1)]
        region, width = ((28, 8), (36, 8), (0, 1)), (4, 4, 1)
        centre = (30.0, 22.0, 0.0)
    elif num_dim == 3:
        dims = (24, 24, 24)
        hole_boxes = [((4, 7), (4, 7), (4, 7)), ((13, 16), (13, 16), (13, 16)),
                      ((0, 3), (13, 16), (0, 2)), ((0, 3), (13, 16), (21, 23)),
                      ((20, 23), (0, 2), (0, 3)), ((20, 23), (21, 23), (20, 23))]
        recv_boxes = [((11, 12), (13, 16), (13, 16)), ((17, 18), (13, 16), (13, 16)),
                      ((13, 16), (11, 12), (13, 16)), ((13, 16), (17, 18), (13, 16)),
                      ((13, 16), (13, 16), (11, 12)), ((13, 16), (13, 16), (17, 18)),
                      ((0, 3), (13, 16), (19, 20)), ((20, 23), (19, 20), (20, 23))]
        region, width = ((8, 5), (18, 3), (4, 5)), (4, 4, 4)
        centre = (11.0, 12.0, 12.0)
    else:
        raise ValueError("num_dim must be 2 or 3")
    nx, ny, nz = dims
    hole = _boxes_mask(dims, hole_boxes)
    recv = _boxes_mask(dims, recv_boxes) & ~hole
    c = [np.arange(n, dtype=np.float64) for n in dims]
    zz, yy, xx = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    mean = np.zeros((5,) + xx.shape)
    mean[1], mean[2] = 0.3, 0.2
    if num_dim == 3:
        mean[3] = 0.1
    mean[4] = 1.0 / gamma
    state = np.zeros((5,) + xx.shape)
    r2 = (xx - centre[0]) ** 2 + (yy - centre[1]) ** 2 + (zz - centre[2]) ** 2
    state[4] = 1e-3 * _gauss(r2, 6.0)
    state[1] = 2e-4 * _gauss(r2, 8.0)
    blk = Block(xx, yy, zz if num_dim == 3 else np.zeros_like(xx), mean, state)
    kk, jj, ii = np.nonzero(recv)
    order = np.lexsort((ii, jj, kk))  # i fastest
    ii, jj, kk = ii[order], jj[order], kk[order]
    (ri, rn), (rj, rm), (rk, rl) = region
    donor = np.stack([ri + ii % rn, rj + jj % rm, (rk + kk % rl) if num_dim == 3 else np.zeros_like(kk)], axis=1)
    W = width[0] * width[1] * width[2]
    ovs = overset_mod.OversetMap(
        num_dim=num_dim, block_points=[nx * ny * nz], recv_block=np.zeros(ii.size, np.int32),
        recv_ijk=np.stack([ii, jj, kk], axis=1).astype(np.int32), donor_block=np.zeros(ii.size, np.int32),
        donor_ijk=donor.astype(np.int32), width=width, weights=rng.uniform(0.5, 1.5, size=(ii.size, W)),
        hole_block=np.zeros(int(hole.sum()), np.int32), hole_ijk=_hole_ijk(hole))
    return Case(name=f"holes{num_dim}d", num_dim=num_dim, blocks=[blk], gamma=gamma, nsteps=nsteps,
                overset=ovs, notes=f"{num_dim}-D block {dims} with hand-set holes and receivers")


def _hole_ijk(hole: np.ndarray) -> np.ndarray:
    kk, jj, ii = np.nonzero(hole)
    order = np.lexsort((ii, jj, kk))
    return np.stack([ii[order], jj[order], kk[order]], axis=1).astype(np.int32)


def with_scalars(case: Case, n: int = 2, seed: int = 21, amplitude: float = 1e-2) -> Case:
    """``case`` with ``n`` passive scalars (PHYSICAL_MODEL = LEE_SCALAR): on every block mean
    fields Z_bar_k = 1 + 0.5 tanh((x cos a_k + y sin a_k) / L) with seed-drawn directions a_k
    (L a quarter of the domain's extent, so that grad Z_bar is non-zero and varies), and Gaussian
    blobs Z_k' of ``amplitude`` at seed-drawn centres, zero in holes. The reference runs
    LEE_SCALAR under SIMULATION = CASE_LINEAR_NOZZLE, whose branch of
    source::apply_physicalSource adds nothing, so the case's monopole is dropped."""
    if case.simulation != "CASE_KBK_COMBUSTOR":
        raise ValueError("LEE_SCALAR runs under CASE_LINEAR_NOZZLE: the case's own source would be lost")
    case.monopole = None
    rng = np.random.default_rng(seed)
    xs = np.concatenate([b.x.ravel() for b in case.blocks])
    ys = np.concatenate([b.y.ravel() for b in case.blocks])
    zs = np.concatenate([b.z.ravel() for b in case.blocks])
    ext = max(np.ptp(xs), np.ptp(ys), 1e-12)
    L = 0.25 * ext
    ang = rng.uniform(0.0, 2.0 * math.pi, size=n)
    centres = [(rng.uniform(xs.min(), xs.max()), rng.uniform(ys.min(), ys.max()), rng.uniform(zs.min(), zs.max()))
               for _ in range(n)]
    hw = 0.15 * ext
    for blk in case.blocks:
        zm = np.empty((n,) + blk.x.shape)
        zq = np.empty((n,) + blk.x.shape)
        for k in range(n):
            zm[k] = 1.0 + 0.5 * np.tanh((blk.x * math.cos(ang[k]) + blk.y * math.sin(ang[k])) / L)
            cx, cy, cz = centres[k]
            r2 = (blk.x - cx) ** 2 + (blk.y - cy) ** 2 + (case.num_dim == 3) * (blk.z - cz) ** 2
            zq[k] = amplitude * _gauss(r2, hw)
        if blk.iblank is not None:
            zq[:, blk.iblank == 1] = 0.0
        blk.zmean, blk.zstate = zm, zq
    case.name += f"_scalars{n}"
    return case
