"""PLOT3D whole-multiblock files and camille's text inputs (deck and BC file).

File layouts follow the reference's serial readers and writers:

* grid ``.xyz`` (src/io/plot3d.cpp:183-223, 443-520): int32 nblocks, then
  int32 (nxi, neta, nzeta) per block, then per block x, y, z as float64 arrays,
  i fastest. Always three coordinates, also in 2-D (z = 0).
* solution ``.q`` (src/io/plot3d.cpp:715-835): the same header, then per block
  float64 tau[4] = {0, 1, step, time} followed by nvar fields.
* function ``.q`` (src/io/plot3d.cpp:881-989): per-block header int32
  (nxi, neta, nzeta, nvar), then per block nvar fields.
* deck ``camille.in`` (src/io/io.cpp:567-625, src/core/input.cpp:99-284): one
  ``KEY = value[, SUBKEY = value...]`` per line.
* BC file (src/io/io.cpp:957-1272): nine columns ``iblock type +-dir is ie js je ks ke``;
  a leading ``-`` on an index counts from the block's last index.

Arrays here are numpy arrays shaped (nzeta, neta, nxi) (or (nvar, nzeta, neta, nxi)),
so C order is the reference's idx1D order (src/geometry/geometry.h:131-136).
"""
from __future__ import annotations

import numpy as np

_I4 = np.dtype("<i4")
_F8 = np.dtype("<f8")


def write_grid(path: str, blocks: list[tuple[np.ndarray, np.ndarray, np.ndarray]]) -> None:
    with open(path, "wb") as f:
        np.array([len(blocks)], _I4).tofile(f)
        for x, _, _ in blocks:
            nz, ny, nx = x.shape
            np.array([nx, ny, nz], _I4).tofile(f)
        for x, y, z in blocks:
            for c in (x, y, z):
                np.ascontiguousarray(c, _F8).tofile(f)


def write_solution(path: str, fields: list[np.ndarray], step: int = 0, time: float = 0.0) -> None:
    with open(path, "wb") as f:
        np.array([len(fields)], _I4).tofile(f)
        for q in fields:
            _, nz, ny, nx = q.shape
            np.array([nx, ny, nz], _I4).tofile(f)
        for q in fields:
            np.array([0.0, 1.0, float(step), float(time)], _F8).tofile(f)
            np.ascontiguousarray(q, _F8).tofile(f)


def write_function(path: str, fields: list[np.ndarray]) -> None:
    with open(path, "wb") as f:
        np.array([len(fields)], _I4).tofile(f)
        for q in fields:
            nv, nz, ny, nx = q.shape
            np.array([nx, ny, nz, nv], _I4).tofile(f)
        for q in fields:
            np.ascontiguousarray(q, _F8).tofile(f)


def read_grid(path: str) -> list[tuple[np.ndarray, np.ndarray, np.ndarray]]:
    with open(path, "rb") as f:
        nb = int(np.fromfile(f, _I4, 1)[0])
        dims = np.fromfile(f, _I4, 3 * nb).reshape(nb, 3)
        out = []
        for nx, ny, nz in dims:
            n = int(nx) * int(ny) * int(nz)
            xyz = np.fromfile(f, _F8, 3 * n).reshape(3, nz, ny, nx)
            out.append((xyz[0], xyz[1], xyz[2]))
    return out


def read_solution(path: str, nvar: int = 5) -> tuple[list[np.ndarray], list[np.ndarray]]:
    with open(path, "rb") as f:
        nb = int(np.fromfile(f, _I4, 1)[0])
        dims = np.fromfile(f, _I4, 3 * nb).reshape(nb, 3)
        qs, taus = [], []
        for nx, ny, nz in dims:
            taus.append(np.fromfile(f, _F8, 4))
            n = int(nx) * int(ny) * int(nz)
            qs.append(np.fromfile(f, _F8, nvar * n).reshape(nvar, nz, ny, nx))
    return qs, taus


def read_function(path: str) -> list[np.ndarray]:
    with open(path, "rb") as f:
        nb = int(np.fromfile(f, _I4, 1)[0])
        dims = np.fromfile(f, _I4, 4 * nb).reshape(nb, 4)
        out = []
        for nx, ny, nz, nv in dims:
            n = int(nx) * int(ny) * int(nz)
            out.append(np.fromfile(f, _F8, int(nv) * n).reshape(nv, nz, ny, nx))
    return out


def write_deck(path: str, lines: list[str]) -> None:
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_bc(path: str, lines: list[str]) -> None:
    with open(path, "w") as f:
        f.write("# iblock type dir is ie js je ks ke\n")
        for ln in lines:
            f.write(ln + "\n")
