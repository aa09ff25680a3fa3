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

from . import plot3d

BC_TYPES = {
    "sponge_freund_ambient": 1000,
    "neumann": 100,
    "wall_slip_kinematic": 201,
}
DIRS = {"XI": 0, "ETA": 1, "ZETA": 2}


@dataclasses.dataclass
class Block:
    x: np.ndarray          # (nz, ny, nx) float64
    y: np.ndarray
    z: np.ndarray
    mean: np.ndarray       # (5, nz, ny, nx): s_bar, u_bar, v_bar, w_bar, p_bar
    state: np.ndarray      # (5, nz, ny, nx): s', u', v', w', p'
    iblank: Optional[np.ndarray] = None  # (nz, ny, nx) int32: 0 fluid, 1 hole, -1 receiver

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
    notes: str = ""

    @property
    def npoints(self) -> int:
        return sum(b.npoints for b in self.blocks)

    # ---- reference input files -------------------------------------------------
    def deck_lines(self, dt: Optional[float], nsteps: int, grid: str, mean: str, bc: str) -> list[str]:
        fix = "FIX_DT" if dt is not None else "FIX_CFL"
        lines = [
            f"DIMENSION = {self.num_dim}",
            "AXISYMMETRY = FALSE",
            "PHYSICAL_MODEL = LEE",
            "FLUID_MODEL = IDEAL_GAS_CALORIC",
            "SIMULATION = CASE_KBK_COMBUSTOR",
            f"GAMMA_SPECIFICHEAT = {self.gamma!r}",
            f"FIX_DT_OR_CFL = {fix}",
            f"DT = {dt!r}" if dt is not None else "DT = 1.0E-6",
            f"CFL = {self.cfl!r}",
            f"TEMPORAL_SCHEME = {self.rk}",
            f"NUM_TOTAL_TIMESTEP = {nsteps}",
            "REPORT_TIMESTEP = 2000000000",
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
            "OVERSET = NONE",
            "DOMAIN_DECOMPOSITION = DECOMP_1D",
            "FILE_FORMAT = PLOT3D",
            f"GRID_FILE = {grid}",
            f"BASESTATE_FILE = {mean}",
            f"BC_FILE = {bc}",
            "SOLUTION_WRITING_TIME = 1.0E+300",
            "HARMONIC_WAVE = NONE",
            "INTERPOLATE_SOLUTION = NONE",
        ]
        return lines

    def write_reference_inputs(self, workdir: str, dt: Optional[float], nsteps: int,
                               step: int = 0, time: float = 0.0) -> str:
        """Write grid, mean, restart, BC and deck files; return the restart path."""
        os.makedirs(workdir, exist_ok=True)
        grid, mean, ic, bc = (os.path.join(workdir, n) for n in ("grid.xyz", "mean.q", "ic.q", "bc.in"))
        plot3d.write_grid(grid, [(b.x, b.y, b.z) for b in self.blocks])
        plot3d.write_function(mean, [b.mean for b in self.blocks])
        plot3d.write_solution(ic, [b.state for b in self.blocks], step=step, time=time)
        plot3d.write_bc(bc, [bd.line() for bd in self.boundaries])
        plot3d.write_deck(os.path.join(workdir, "camille.in"), self.deck_lines(dt, nsteps, grid, mean, bc))
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
