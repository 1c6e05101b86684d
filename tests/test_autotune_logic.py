"""Autotuner helpers on the CPU: radix-order candidates multiply to the transform length,
start with the library's default order (radix 8 while possible, then 4, 2, 7, 5, 3,
larger odd factors), use register radices only and are distinct; the per-member
ensemble tile rule h = B = clamp(c // N, 2, 16)."""
import math

from fastiso_b200.autotune import REG_RADICES, default_schedule, rule_tiles, schedule_candidates


def test_default_schedule_matches_the_library_order():
    assert default_schedule(350) == [2, 7, 5, 5]
    assert default_schedule(1024) == [8, 8, 8, 2]
    assert default_schedule(256) == [8, 8, 4]
    assert default_schedule(700) == [4, 7, 5, 5]
    assert default_schedule(96) == [8, 4, 3]
    assert default_schedule(121) == [11, 11]
    assert default_schedule(13) == [13]


def test_candidates_are_factorisations():
    for L in (64, 96, 128, 192, 256, 350, 700, 1024, 2048, 121):
        c = schedule_candidates(L, limit=12)
        assert c[0] == default_schedule(L)
        assert len({tuple(x) for x in c}) == len(c)
        for sched in c:
            assert math.prod(sched) == L
            assert all(r in REG_RADICES for r in sched) or sched == default_schedule(L)


def test_rule_tiles():
    assert rule_tiles(2048, 64) == (16, 16)
    assert rule_tiles(2048, 192) == (10, 10)
    assert rule_tiles(2048, 256) == (8, 8)
    assert rule_tiles(2048, 1024) == (2, 2)
    assert rule_tiles(2048, 4096) == (2, 2)
