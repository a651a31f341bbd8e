"""The round schedule of the culling pair kernel (openmm-rs_b200/csrc/pair.cu, pair_kernel_cull),
modelled on the host: the kernel's warp-uniform decisions over one run of tiles, replayed for
random and adversarial patterns of kept entries.

Per half of block I the kernel keeps a ring of kRing = 64 entries in shared memory: kept
entries are written after the tail, a round takes 16 from each head (topping a half with fewer
up with dummies written after its tail) and advances both heads by 16.  Before a tile's entries
are appended, rounds run while both halves hold 16 or either holds more than kRing - 16; before
a self or minimum-image tile, and at the end of the run, the queue is drained.  The model checks
what the kernel relies on but cannot check itself: no write lands on a queued entry, no ring
holds more than kRing entries, every kept entry is evaluated in exactly one round, and dummies
fill exactly the places kept entries leave empty.
"""
import numpy as np
import pytest

K_RING = 64


class Ring:
    """One half's ring: slot contents (None = free), head and tail counters."""

    def __init__(self):
        self.slot = [None] * K_RING
        self.head = 0
        self.tail = 0

    def put(self, pos, item):
        k = pos % K_RING
        assert self.slot[k] is None, "a write landed on a queued entry"
        self.slot[k] = item


def run_schedule(tiles):
    """tiles: list of ('keep', n0, n1) (kept entries per half) or ('special',).
    Returns the entries each round evaluated and the number of dummies written."""
    halves = [Ring(), Ring()]
    seen, dummies, next_id = [], 0, 0

    def queue_round():
        nonlocal dummies
        for r in halves:  # top up to 16 after the tail
            q = r.tail - r.head
            assert q >= 0
            for e in range(q, 16):
                r.put(r.head + e, "dummy")
                dummies += 1
        for h, r in enumerate(halves):  # the round reads 16 from the head and frees them
            for e in range(16):
                k = (r.head + e) % K_RING
                item = r.slot[k]
                assert item is not None
                if item != "dummy":
                    seen.append(item)
                r.slot[k] = None
            r.head += 16
            r.tail = max(r.tail, r.head)
            assert r.head % 16 == 0

    def drain():
        while any(r.tail > r.head for r in halves):
            queue_round()

    for tile in tiles:
        if tile[0] == "special":  # self or minimum-image tile: the queue is drained first
            drain()
            assert all(r.tail == r.head for r in halves)
            continue
        counts = tile[1:]
        for h, r in enumerate(halves):
            assert r.tail - r.head + counts[h] <= K_RING, "ring overflow"
            for i in range(counts[h]):
                r.put(r.tail + i, (h, next_id))
                next_id += 1
            r.tail += counts[h]
        q0, q1 = (r.tail - r.head for r in halves)
        while q0 >= 16 and q1 >= 16:
            queue_round()
            q0, q1 = (r.tail - r.head for r in halves)
        while q0 > K_RING - 16 or q1 > K_RING - 16:
            queue_round()
            q0, q1 = (r.tail - r.head for r in halves)
    drain()
    return seen, dummies, next_id


def patterns():
    rng = np.random.default_rng(5)
    yield "all kept", [("keep", 16, 16)] * 40
    yield "one half empty", [("keep", 16, 0)] * 40
    yield "alternating halves", [("keep", 16, 0), ("keep", 0, 16)] * 20
    yield "nothing kept", [("keep", 0, 0)] * 10
    yield "specials between", [("special",), ("keep", 15, 3), ("special",), ("keep", 1, 16)] * 8
    for s in range(20):
        tiles = []
        for _ in range(int(rng.integers(1, 70))):
            if rng.random() < 0.05:
                tiles.append(("special",))
            else:
                tiles.append(("keep", int(rng.integers(0, 17)), int(rng.integers(0, 17))))
        yield f"random {s}", tiles


@pytest.mark.parametrize("name,tiles", list(patterns()), ids=[p[0] for p in patterns()])
def test_culling_round_schedule_keeps_the_ring_consistent(name, tiles):
    seen, dummies, n_kept = run_schedule(tiles)
    # every kept entry is evaluated exactly once
    assert len(seen) == len(set(seen)) == n_kept
    # rounds evaluate 16 places per half; dummies fill exactly what kept entries leave
    assert (n_kept + dummies) % 32 == 0
