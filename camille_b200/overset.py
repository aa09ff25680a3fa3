"""Overset donor maps: the hole cut, the receiver fringe, explicit Lagrange donor stencils and
camille's Overture overset file.

camille reads its donor maps from a binary file written by Overture (an external grid
generator that is not part of camille) in the layout of ``read_overset_at_headrank``
(camille src/io/overture.cpp:473-680), all little-endian int32 / float64:

    int num_dim
    int num_blocks
    int num_cells[num_blocks]                    (points per block)
    int num_receivers[num_blocks]
    int receiver_block[R]                        (R = sum of num_receivers)
    int receiver_ijk[R][num_dim]                 (block-level, 0-based)
    int donor_block[R]
    int donor_ijk[R][num_dim]                    (lower-left corner of the donor stencil)
    per block: int width[3]; then, for each of that block's receivers, width[0]*width[1]*width[2]
               float64 weights, zeta outermost and xi innermost
    int num_holes[num_blocks]
    int hole_ijk[sum of num_holes][3]

Receivers are grouped by block in block order. The reference takes width - 1 as the
interpolation order (``OVERSET ... ORDER_ACCURACY``, overture.cpp:609), normalises each
receiver's weights by their sum (src/overset/overset.cpp:516-526), marks holes BLANKED and
receivers INTERPOLATED (:683-790) and, after every boundary update, overwrites each receiver
with the weighted sum of its donor stencil (:886-974, :1241-1278).

This module is the donor tool camille lacks: it cuts holes, picks the receiver fringe and
computes tensor-product Lagrange weights in the donor grid's computational coordinates from
analytic inverses of the grid mappings. Both the CUDA library and the CPU oracle consume the
file it writes, so donor generation itself has no reference to agree with.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional, Sequence

import numpy as np

BLANKED, INTERPOLATED, NOTBLANKED = 1, -1, 0


@dataclasses.dataclass
class OversetMap:
    num_dim: int
    block_points: list[int]         # points per block
    recv_block: np.ndarray          # (R,) int32, grouped by block in block order
    recv_ijk: np.ndarray            # (R, 3) int32
    donor_block: np.ndarray         # (R,) int32
    donor_ijk: np.ndarray           # (R, 3) int32, lower-left corner of the stencil
    width: tuple[int, int, int]     # stencil points per direction (1 in unused directions)
    weights: np.ndarray             # (R, width[2]*width[1]*width[0]) float64, xi fastest
    hole_block: np.ndarray          # (H,) int32, grouped by block
    hole_ijk: np.ndarray            # (H, 3) int32

    @property
    def num_receivers(self) -> int:
        return int(self.recv_block.size)

    @property
    def order(self) -> int:
        return self.width[0] - 1

    def write(self, path: str) -> None:
        nb = len(self.block_points)
        nd = self.num_dim
        counts = np.bincount(self.recv_block, minlength=nb).astype("<i4")
        if np.any(np.diff(self.recv_block) < 0):
            raise ValueError("receivers must be grouped by block in block order")
        holes = np.bincount(self.hole_block, minlength=nb).astype("<i4") if self.hole_block.size else \
            np.zeros(nb, "<i4")
        if self.hole_block.size and np.any(np.diff(self.hole_block) < 0):
            raise ValueError("holes must be grouped by block in block order")
        with open(path, "wb") as f:
            np.array([nd, nb], "<i4").tofile(f)
            np.asarray(self.block_points, "<i4").tofile(f)
            counts.tofile(f)
            self.recv_block.astype("<i4").tofile(f)
            self.recv_ijk[:, :nd].astype("<i4").tofile(f)
            self.donor_block.astype("<i4").tofile(f)
            self.donor_ijk[:, :nd].astype("<i4").tofile(f)
            start = 0
            for b in range(nb):
                np.asarray(self.width, "<i4").tofile(f)
                self.weights[start:start + counts[b]].astype("<f8").tofile(f)
                start += int(counts[b])
            holes.tofile(f)
            self.hole_ijk.astype("<i4").reshape(-1, 3).tofile(f)

    @classmethod
    def read(cls, path: str) -> "OversetMap":
        with open(path, "rb") as f:
            nd, nb = (int(v) for v in np.fromfile(f, "<i4", 2))
            pts = [int(v) for v in np.fromfile(f, "<i4", nb)]
            counts = np.fromfile(f, "<i4", nb)
            R = int(counts.sum())
            rb = np.fromfile(f, "<i4", R)
            rijk = np.zeros((R, 3), np.int32)
            rijk[:, :nd] = np.fromfile(f, "<i4", R * nd).reshape(R, nd)
            db = np.fromfile(f, "<i4", R)
            dijk = np.zeros((R, 3), np.int32)
            dijk[:, :nd] = np.fromfile(f, "<i4", R * nd).reshape(R, nd)
            wts, width = [], (1, 1, 1)
            for b in range(nb):
                width = tuple(int(v) for v in np.fromfile(f, "<i4", 3))
                W = width[0] * width[1] * width[2]
                wts.append(np.fromfile(f, "<f8", int(counts[b]) * W).reshape(-1, W))
            holes = np.fromfile(f, "<i4", nb)
            H = int(holes.sum())
            hijk = np.fromfile(f, "<i4", 3 * H).reshape(H, 3)
        hb = np.repeat(np.arange(nb, dtype=np.int32), holes)
        return cls(nd, pts, rb.astype(np.int32), rijk, db.astype(np.int32), dijk, width,
                   np.concatenate(wts) if wts else np.zeros((0, 1)), hb, hijk.astype(np.int32))

    def normalised_weights(self) -> np.ndarray:
        """The weights as the reference holds them after initialize_donor (overset.cpp:516-526):
        each row times 1 / (its sum accumulated left to right)."""
        out = np.empty_like(self.weights)
        for r in range(self.weights.shape[0]):
            s = 0.0
            for w in self.weights[r]:
                s += float(w)
            inv = 1.0 / s
            out[r] = [float(w) * inv for w in self.weights[r]]
        return out


def lagrange_weights(u: float, n: int = 4) -> list[float]:
    """n-point Lagrange basis at nodes 0..n-1, evaluated at u."""
    out = []
    for a in range(n):
        v = 1.0
        for b in range(n):
            if b != a:
                v *= (u - b) / (a - b)
        out.append(v)
    return out


@dataclasses.dataclass
class DonorGrid:
    """A 2-D block seen as a donor: its dimensions, an inverse mapping from physical (x, y) to
    candidate computational coordinates (xi, eta) (several for a periodic direction), and a
    mask of points that may serve as donors (not holes, not receivers)."""
    dims: tuple[int, int]
    inverse: Callable[[float, float], Sequence[tuple[float, float]]]
    eligible: np.ndarray  # (ny, nx) bool


def find_donor(grid: DonorGrid, x: float, y: float, width: int = 4) -> Optional[tuple[int, int, list[float]]]:
    """Lower-left corner and tensor-product weights (xi fastest) of a width x width stencil of
    eligible points that contains (x, y): centred on the containing cell when that stencil is
    eligible, else shifted by up to width/2 points per direction (the point stays inside the
    stencil, so the weights interpolate); None if no candidate fits."""
    nx, ny = grid.dims
    half = width // 2 - 1
    shifts = sorted(range(-(width // 2), width // 2 + 1), key=lambda v: (abs(v), v))
    for xi, eta in grid.inverse(x, y):
        if not (-1e-9 <= xi <= nx - 1 + 1e-9 and -1e-9 <= eta <= ny - 1 + 1e-9):
            continue
        ci, cj = int(math.floor(xi)) - half, int(math.floor(eta)) - half
        best = None
        for si in shifts:
            for sj in shifts:
                i0 = min(max(ci + si, 0), nx - width)
                j0 = min(max(cj + sj, 0), ny - width)
                tol = 1e-9  # a receiver on a donor grid line comes back within rounding of it
                if not (i0 - tol <= xi <= i0 + width - 1 + tol and j0 - tol <= eta <= j0 + width - 1 + tol):
                    continue
                if grid.eligible[j0:j0 + width, i0:i0 + width].all():
                    cost = abs(i0 - ci) + abs(j0 - cj)
                    if best is None or cost < best[0]:
                        best = (cost, i0, j0)
        if best is None:
            continue
        _, i0, j0 = best
        lx = lagrange_weights(xi - i0, width)
        ly = lagrange_weights(eta - j0, width)
        return i0, j0, [ly[b] * lx[a] for b in range(width) for a in range(width)]
    return None
