"""Host-side check of the served form's staging ring: pieces are taken and
given back first in, first out, and no live piece may overlap another or
run past the buffer, whatever the sizes (random sequences)."""
import collections
import random

import pytest


class _Buf:
    def __init__(self, n):
        self.n = n

    def numel(self):
        return self.n


@pytest.mark.parametrize("size", [4096, 10000, 1 << 16])
def test_ring_pieces_never_overlap(size):
    from flash_map.serve import _Ring

    rng = random.Random(size)
    ring = _Ring(_Buf(size))
    live = collections.deque()
    taken = 0
    for _ in range(20000):
        if live and rng.random() < 0.45:
            ring.give()
            live.popleft()
            continue
        need = rng.randint(1, size // 3)
        off = ring.take(need)
        if off is None:
            assert live  # an empty ring always has room for a piece that fits
            continue
        assert 0 <= off and off + need <= size
        for o, n in live:
            assert off + need <= o or o + n <= off
        live.append((off, need))
        taken += 1
    assert taken > 1000
