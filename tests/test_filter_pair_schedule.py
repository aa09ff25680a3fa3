"""CPU model of the two-point fused filter's plane schedule (camille_b200/csrc/lee_filter_pair.cu).

The kernel keeps a ring of h + 4 TMA slots per CTA: plane p of a chunk lands in slot
(p - plo) mod (h + 4); thread 0 fills the ring at the start and, at the one barrier of each
loaded plane p, issues the planes up to p + 3; a thread reads plane p's slot for its xi pass
(before that barrier) and reads the pre-filter value of plane p - h back from its slot when it
finishes that plane (after the barrier of iteration p, or in the trailing iterations that load
nothing). This model replays that schedule for many block depths, chunks and half-widths and
checks that every plane is issued before it is waited on, and that no slot is re-issued while a
read of its previous plane is still to come; and that a pair's row window (2 HP + 2 points of
8-byte words) lies inside the box row for every thread of the tile.
"""
from __future__ import annotations

import itertools

import pytest

PF = 3
TX = 64


def _box(hf: int):
    hx = ((hf + 3) // 4) * 4
    return hx, TX + 2 * hx


def _chunk_schedule(nz: int, k0: int, k1: int, hf: int) -> None:
    ns = hf + 1 + PF
    plo, phi = max(0, k0 - hf), min(nz - 1, k1 - 1 + hf)
    issued_at = {}                      # plane -> iteration of its issue (-1: the initial fill)
    for q in range(plo, min(phi, plo + ns - 1) + 1):
        issued_at[q] = -1
    next_issue = min(phi, plo + ns - 1) + 1
    last_read = {}                      # plane -> iteration of its last read
    for it, p in enumerate(range(k0 - hf, k1 + hf)):
        if plo <= p <= phi:
            assert p in issued_at, (nz, k0, k1, hf, p)           # waited on only once issued
            last_read[p] = it                                     # xi pass, before the barrier
            # the barrier: every iteration before `it` is complete; issue up to p + PF
            while next_issue <= min(phi, p + PF):
                prev = next_issue - ns                            # the slot's previous plane
                if prev >= plo:
                    assert last_read.get(prev, -1) < it, (nz, k0, k1, hf, next_issue, prev)
                issued_at[next_issue] = it
                next_issue += 1
        kf = p - hf
        if k0 <= kf < k1:
            # the pre-filter value of plane kf from its slot, after this iteration's barrier
            assert kf + ns not in issued_at or issued_at[kf + ns] > it, (nz, k0, k1, hf, kf)
            last_read[kf] = it
    assert next_issue == phi + 1


@pytest.mark.parametrize("hf", [2, 4, 5])
def test_ring_slots_are_reissued_only_after_their_last_read(hf):
    for nz in (2 * hf + 1, 16, 37, 64, 255, 256):
        for chunk in sorted({8, 11, 16, 29, 32, 43, 64, 86, 96, 128, 256, (nz + 2) // 3}):
            for k0 in range(0, nz, chunk):
                _chunk_schedule(nz, k0, min(nz, k0 + chunk), hf)


@pytest.mark.parametrize("hf", [2, 4, 5])
def test_pair_row_windows_lie_inside_the_box(hf):
    hx, bx = _box(hf)
    hp = (hf + 1) // 2
    nw = 1 + 2 * hp
    assert hx % 2 == 0 and bx % 2 == 0  # 8-byte words start on even columns
    for tx in range(TX // 2):
        c = hx + 2 * tx                  # the pair's first point in the box row
        first, last = c - 2 * hp, c - 2 * hp + 2 * nw - 1
        assert first >= 0 and last <= bx - 1 and first % 2 == 0
        for o, lane in itertools.product(range(-hf, hf + 1), (0, 1)):
            assert first <= c + lane + o <= last  # every tap of both points is in the window
