"""Host-side parts of the serving loop: the device arena's address arithmetic
and argument checks.  No GPU is touched (the arena works on any base)."""
import ctypes as C

import numpy as np
import pytest

BASE = 1 << 40
ALIGN = 512


@pytest.fixture
def arena(T):
    h = C.c_void_p()
    assert T.lib.tops_arena_create(BASE, 1 << 20, C.byref(h)) == T.TOPS_OK
    yield h
    T.lib.tops_arena_destroy(h)


def test_arena_alignment_and_accounting(T, arena):
    a = T.lib.tops_arena_alloc(arena, 1)
    b = T.lib.tops_arena_alloc(arena, 1000)
    c = T.lib.tops_arena_alloc(arena, 4096)
    assert a == BASE and b == BASE + ALIGN and c == BASE + 3 * ALIGN
    assert T.lib.tops_arena_in_use(arena) == ALIGN + 2 * ALIGN + 4096
    for p in (a, b, c):
        assert p % ALIGN == 0


def test_arena_first_fit_and_coalescing(T, arena):
    blocks = [T.lib.tops_arena_alloc(arena, 64 * 1024) for _ in range(16)]
    assert all(blocks) and T.lib.tops_arena_alloc(arena, 1) == 0   # full
    # free every other block: 8 holes, none larger than one block
    for p in blocks[::2]:
        assert T.lib.tops_arena_release(arena, p) == T.TOPS_OK
    assert T.lib.tops_arena_free_ranges(arena) == 8
    assert T.lib.tops_arena_largest_free(arena) == 64 * 1024
    assert T.lib.tops_arena_alloc(arena, 128 * 1024) == 0          # fragmented
    assert T.lib.tops_arena_alloc(arena, 32 * 1024) == blocks[0]   # first fit
    # freeing the rest coalesces everything back into one range
    assert T.lib.tops_arena_release(arena, blocks[0]) == T.TOPS_OK
    for p in blocks[1::2]:
        assert T.lib.tops_arena_release(arena, p) == T.TOPS_OK
    assert T.lib.tops_arena_free_ranges(arena) == 1
    assert T.lib.tops_arena_largest_free(arena) == 1 << 20
    assert T.lib.tops_arena_in_use(arena) == 0


def test_arena_rejects_foreign_and_double_release(T, arena):
    p = T.lib.tops_arena_alloc(arena, 100)
    assert T.lib.tops_arena_release(arena, p + ALIGN) == T.TOPS_E_INVALID
    assert T.lib.tops_arena_release(arena, 12345) == T.TOPS_E_INVALID
    assert T.lib.tops_arena_release(arena, p) == T.TOPS_OK
    assert T.lib.tops_arena_release(arena, p) == T.TOPS_E_INVALID


def test_arena_random_churn_keeps_invariants(T, arena):
    rng = np.random.default_rng(3)
    live = {}
    for _ in range(2000):
        if live and rng.random() < 0.45:
            p = list(live)[rng.integers(len(live))]
            assert T.lib.tops_arena_release(arena, p) == T.TOPS_OK
            del live[p]
        else:
            n = int(rng.integers(1, 40000))
            p = T.lib.tops_arena_alloc(arena, n)
            if p:
                r = -(-n // ALIGN) * ALIGN
                for q, m in live.items():          # no overlap with live blocks
                    assert p + r <= q or q + m <= p
                live[p] = r
        assert T.lib.tops_arena_in_use(arena) == sum(live.values())
    for p in list(live):
        T.lib.tops_arena_release(arena, p)
    assert T.lib.tops_arena_free_ranges(arena) == 1


def test_server_argument_checks(T):
    h = C.c_void_p()
    bad = T.ServerCfg(1 << 20, 0)
    assert T.lib.tops_server_create(C.byref(bad), C.byref(h)) == T.TOPS_E_INVALID
    bad = T.ServerCfg(100, 2)
    assert T.lib.tops_server_create(C.byref(bad), C.byref(h)) == T.TOPS_E_INVALID
    assert T.lib.tops_server_submit(None, None, None) == T.TOPS_E_INVALID
    assert T.lib.tops_server_job_footprint(None) == 0
    h = C.c_void_p()
    assert T.lib.tops_arena_create(BASE + 3, 1 << 20, C.byref(h)) == T.TOPS_E_INVALID


def test_job_footprint_matches_plan_footprint(T, scene_small):
    S = scene_small
    d = T.JobDesc()
    d.master, d.slave = S.swath[0], S.swath[1]
    d.opts = T.pair_opts()
    fp = T.lib.tops_server_job_footprint(C.byref(d))
    assert fp == T.Pair.footprint(S.swath[0], (0, 0))
    L, W, nb = S.cfg.lines_per_burst, S.cfg.samples_per_burst, S.cfg.n_bursts
    assert fp > nb * L * W * (4 + 4 + 8 + 8 + 4)   # SLCs, ReSlave, ReSlaveESD, coherence


def test_sub_swath_description(T, scene_esd):
    S = scene_esd
    m = S.swath[0]
    sub = T.sub_swath(m, 1, 2)
    assert sub.n_bursts == 2
    assert sub.burst_first_line_time[0] == m.burst_first_line_time[1]
    assert sub.burst_last_line_time[1] == m.burst_last_line_time[2]
    assert sub.fm_list[0].aztime == m.fm_list[1].aztime
    assert sub.n_fm == m.n_fm - 1
