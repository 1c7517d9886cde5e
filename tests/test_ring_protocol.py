"""Host model of the single-window kernel's draw ring (csrc/sweep_window.cu): the producer warp
writes the walker's draws 32 at a time into a 64-entry ring when the walker's published
consumed count leaves room for a batch; the walker publishes its draw index only when it has
entered a new batch of 32 (from the rare branch at the top of an attempt), waits when it needs a
draw beyond hq + 4 that is not yet produced, and moves on by one draw (a site that bounded()
rejected), or by one or two (an attempt that did or did not consume the acceptance uniform).

The model checks, over random and adversarial draw sequences, the two properties the kernel's
bounded waits rely on: every wait of the walker can end (the producer always has room to
produce the draws the walker waits for), and the producer never overwrites a record the walker
can still read (every overwritten draw index lies below the published count, and the walker reads
only draws at or after its current index).  No GPU is involved."""
from __future__ import annotations

import random
import re
from pathlib import Path

SOURCE = Path(__file__).resolve().parents[1] / "replica_exchange_wang_landau_b200" / "csrc" / "sweep_window.cu"


def _ring_size() -> int:
    m = re.search(r"constexpr int kWindowRing = (\d+);", SOURCE.read_text())
    assert m, "kWindowRing not found"
    return int(m.group(1))


BATCH = 32  # the producer's batch: one draw per lane


class Ring:
    def __init__(self, size: int):
        self.size = size
        self.produced = 0
        self.consumed = 0  # the count the walker last published

    def produce_all_room(self) -> None:
        """The producer's loop: a batch whenever produced + 32 - consumed <= ring size."""
        while self.produced + BATCH - self.consumed <= self.size:
            overwritten_top = self.produced + BATCH - 1 - self.size  # highest draw index whose slot is reused
            assert overwritten_top < self.consumed, "producer overwrote a record the walker may still read"
            self.produced += BATCH


def walk(steps: int, moves, ring_size: int) -> int:
    """Runs the walker against the producer; `moves` yields 'reject', 1 or 2 per step."""
    ring = Ring(ring_size)
    ring.produce_all_room()
    hq = published = 0
    waits = 0
    for _, move in zip(range(steps), moves):
        if (hq ^ published) >= BATCH:  # the rare branch publishes the count
            ring.consumed = published = hq
        if hq + 4 >= ring.produced:  # the walker waits for draws [0, hq + 4]
            waits += 1
            ring.produce_all_room()
            assert hq + 4 < ring.produced, f"wait at hq={hq} can never end (produced {ring.produced})"
        # the walker reads draws hq .. hq + 4 only; all must still be in the ring
        assert hq + 4 < ring.produced and hq >= ring.produced - ring_size
        hq += 1 if move == "reject" else move
        ring.produce_all_room()
    return waits


def test_ring_size_matches_kernel():
    assert _ring_size() == 64


def test_random_runs_never_deadlock_or_overwrite():
    size = _ring_size()
    rng = random.Random(5)
    for trial in range(40):
        p_reject = [0.0, 0.01, 0.3][trial % 3]

        def moves():
            while True:
                yield "reject" if rng.random() < p_reject else rng.choice([1, 2])

        walk(20000, moves(), size)


def test_adversarial_runs():
    size = _ring_size()
    # long bursts of rejected site draws, and runs of two-draw attempts only or one-draw only
    for pattern in (["reject"] * 200 + [2] * 50, [2], [1], [1, "reject"], ["reject", "reject", 2]):
        def moves(p=pattern):
            while True:
                yield from p

        walk(5000, moves(), size)


def test_a_ring_without_room_for_two_batches_would_deadlock():
    # the model is not vacuous: with one batch of room the walker's waits cannot end
    def moves():
        while True:
            yield 1

    try:
        walk(100, moves(), BATCH)
    except AssertionError:
        return
    raise AssertionError("expected the model to find a wait that cannot end")
