"""CPU model of the persistent batched step's grid barrier (grid_barrier in
camille_b200/csrc/lee_batch.cu): a counter gb[0] and a generation gb[1], both zero at launch; a
CTA reads the generation, arrives on the counter; the last arrival resets the counter and bumps
the generation, the others spin until the generation moves or their wait limit runs out, in which
case they record the failure and leave the kernel.

CTAs are generators stepped in seeded random orders (each yield is a point where another CTA may
run). The checks: no CTA leaves barrier n before every CTA has arrived at it, successive barriers
reuse the counter correctly, and when the limit runs out (a CTA that stopped early, or a limit of
zero) every CTA leaves the kernel with the failure recorded -- none spins for ever."""
from __future__ import annotations

import random

import pytest


class Dev:
    def __init__(self):
        self.count = 0
        self.gen = 0
        self.err = 0


def cta(dev: Dev, nblk: int, nbar: int, limit: int, log: list, me: int, stop_after: int = -1):
    """One CTA: nbar phases, each followed by a barrier; `limit` spins before giving up (0: at
    once, as a wait limit of 0 does); stop_after >= 0 leaves before that barrier (a CTA that failed)."""
    for b in range(nbar):
        yield
        if b == stop_after:
            dev.err = 1
            log.append(("exit", me, b))
            return
        g = dev.gen
        yield
        arrived = dev.count
        dev.count += 1  # atomicAdd
        log.append(("arrive", me, b))
        yield
        if arrived == nblk - 1:
            dev.count = 0
            yield
            dev.gen += 1
        else:
            ok = limit > 0
            spins = 0
            while ok and dev.gen == g:
                spins += 1
                if spins > limit:
                    ok = False
                yield
            if not ok:
                dev.err = 1
                log.append(("exit", me, b))
                return
        log.append(("leave", me, b))
    log.append(("done", me, nbar))


def run(nblk, nbar, limit, seed, stop=None):
    dev, log = Dev(), []
    gens = [cta(dev, nblk, nbar, limit, log, i, stop[i] if stop else -1) for i in range(nblk)]
    live = list(range(nblk))
    rng = random.Random(seed)
    steps = 0
    while live:
        i = rng.choice(live)
        try:
            next(gens[i])
        except StopIteration:
            live.remove(i)
        steps += 1
        assert steps < 10_000_000, "a CTA spins for ever"
    return dev, log


@pytest.mark.parametrize("seed", range(40))
def test_no_cta_leaves_a_barrier_before_all_arrived(seed):
    nblk, nbar = 2 + seed % 7, 1 + seed % 5
    dev, log = run(nblk, nbar, limit=10**6, seed=seed)
    assert dev.err == 0 and dev.count == 0 and dev.gen == nbar
    arrived = {b: 0 for b in range(nbar)}
    for ev, _, b in log:
        if ev == "arrive":
            arrived[b] += 1
        elif ev == "leave":
            assert arrived[b] == nblk, (seed, b)
    assert sum(1 for ev, _, _ in log if ev == "done") == nblk


@pytest.mark.parametrize("seed", range(20))
def test_a_cta_that_stops_makes_every_cta_give_up(seed):
    nblk, nbar = 3 + seed % 5, 2 + seed % 3
    stop = [-1] * nblk
    stop[seed % nblk] = seed % nbar
    dev, log = run(nblk, nbar, limit=50, seed=seed, stop=stop)
    assert dev.err == 1
    assert not any(ev == "done" for ev, _, _ in log)  # nobody finished the step


@pytest.mark.parametrize("seed", range(10))
def test_a_zero_limit_gives_up_at_once(seed):
    dev, log = run(2 + seed % 6, 3, limit=0, seed=seed)
    assert dev.err == 1
    assert not any(ev == "done" for ev, _, _ in log)
