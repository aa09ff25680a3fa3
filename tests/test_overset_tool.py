"""The donor tool and the Overture overset file (camille_b200/overset.py, cases.cylinder2d).

Donor generation has no reference to agree with (camille reads maps that Overture wrote), so
these tests check the properties the maps must have: the file round-trips, every receiver's
stencil lies inside its donor block on eligible points and contains the receiver, the weights
reproduce the receiver's own coordinates (exactly on the Cartesian background, to
interpolation accuracy on the O-grid), holes and receivers are where the layout puts them, and
the C ABI refuses maps that would read outside a block.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from camille_b200 import api, cases, overset


@pytest.fixture(scope="module")
def small():
    return cases.cylinder2d(nb=64, length=16.0, ntheta=72, nr=24, r_out=3.0, first_cell=0.05, r_cut=1.0, sponge=4,
                            nsteps=2)


def test_file_round_trip(small, tmp_path):
    path = str(tmp_path / "o.bin")
    small.overset.write(path)
    back = overset.OversetMap.read(path)
    o = small.overset
    assert back.num_dim == o.num_dim and back.block_points == o.block_points and back.width == o.width
    for k in ("recv_block", "recv_ijk", "donor_block", "donor_ijk", "weights", "hole_block", "hole_ijk"):
        np.testing.assert_array_equal(getattr(back, k), getattr(o, k))


def test_stencils_interpolate_the_receiver_coordinates(small):
    o = small.overset
    W = o.width[0]
    for r in range(o.num_receivers):
        rb, db = int(o.recv_block[r]), int(o.donor_block[r])
        rblk, dblk = small.blocks[rb], small.blocks[db]
        i, j, _ = o.recv_ijk[r]
        i0, j0, _ = o.donor_ijk[r]
        xs = dblk.x[0, j0:j0 + W, i0:i0 + W].ravel()
        ys = dblk.y[0, j0:j0 + W, i0:i0 + W].ravel()
        w = o.weights[r]
        assert abs(w.sum() - 1.0) < 1e-13
        ex = abs(float(w @ xs) - float(rblk.x[0, j, i]))
        ey = abs(float(w @ ys) - float(rblk.y[0, j, i]))
        tol = 1e-12 if db == 0 else 2e-3  # linear map on the background; r cos(theta) on the O-grid
        assert ex <= tol and ey <= tol, (r, rb, db, ex, ey)


def test_stencils_use_eligible_points_only(small):
    o = small.overset
    W = o.width[0]
    ib = []
    for b, blk in enumerate(small.blocks):
        a = np.zeros(blk.x.shape[1:], np.int32)
        for q in np.nonzero(o.hole_block == b)[0]:
            a[o.hole_ijk[q, 1], o.hole_ijk[q, 0]] = overset.BLANKED
        for q in np.nonzero(o.recv_block == b)[0]:
            a[o.recv_ijk[q, 1], o.recv_ijk[q, 0]] = overset.INTERPOLATED
        ib.append(a)
    for r in range(o.num_receivers):
        i0, j0, _ = o.donor_ijk[r]
        st = ib[int(o.donor_block[r])][j0:j0 + W, i0:i0 + W]
        assert st.shape == (W, W) and np.all(st == overset.NOTBLANKED)
    # the background is blanked inside r_cut, receivers ring the hole, and the O-grid's
    # receivers are its outer rings and its seam lines
    bg = small.blocks[0]
    r_bg = np.hypot(bg.x[0], bg.y[0])
    assert np.all((ib[0] == overset.BLANKED) == (r_bg < 1.0))
    assert np.all(ib[1][-2:, :] == overset.INTERPOLATED)
    assert np.all(ib[1][:, :2] == overset.INTERPOLATED) and np.all(ib[1][:, -2:] == overset.INTERPOLATED)


def test_seam_receivers_are_self_donated(small):
    o = small.overset
    seam = (o.recv_block == 1) & (o.recv_ijk[:, 1] < 22)
    assert seam.any() and np.all(o.donor_block[seam] == 1)
    outer = (o.recv_block == 1) & (o.recv_ijk[:, 1] >= 22)
    assert np.all(o.donor_block[outer] == 0)


def test_normalised_weights_match_the_reference_rule(small, oracle_lib):
    s = api.Solver(oracle_lib, small)
    np.testing.assert_array_equal(s.get_overset()["weights"], small.overset.normalised_weights())


def test_abi_refuses_a_stencil_outside_its_block(small, oracle_lib):
    """A donor corner whose stencil would run past the block is refused before any run."""
    o = small.overset
    bad = o.donor_ijk.copy()
    bad[0, 0] = small.blocks[int(o.donor_block[0])].dims[0] - 2
    lib = oracle_lib
    cfg = api.config_for(small)
    ctx = C.c_void_p()
    assert lib.create(C.byref(cfg), C.byref(ctx)) == 0
    try:
        for b, blk in enumerate(small.blocks):
            nx, ny, nz = blk.dims
            xs = [np.ascontiguousarray(a) for a in (blk.x, blk.y, blk.z)]
            assert lib.set_block(ctx, b, nx, ny, nz, *[a.ctypes.data_as(C.POINTER(C.c_double)) for a in xs],
                                 None) == 0
        arrs = [np.ascontiguousarray(a, np.int32) for a in (o.recv_block, o.recv_ijk, o.donor_block, bad,
                                                            np.asarray(o.width), o.hole_block, o.hole_ijk)]
        w = np.ascontiguousarray(o.weights)
        rc = lib.set_overset(ctx, o.num_receivers, *[a.ctypes.data_as(C.POINTER(C.c_int)) for a in arrs[:5]],
                             w.ctypes.data_as(C.POINTER(C.c_double)), int(o.hole_block.size),
                             arrs[5].ctypes.data_as(C.POINTER(C.c_int)), arrs[6].ctypes.data_as(C.POINTER(C.c_int)))
        assert rc == 1  # LEE_ERR_ARG
        assert b"outside" in lib.last_error(ctx)
    finally:
        lib.destroy(ctx)
