"""CPU: the bookkeeping of the bidirectional tracer's connection-parallel
kernels (dort_b200/csrc/bdpt.cu, bdpt.cuh), restated here to check the
bounds its device writes rely on.

For every max_depth the tracer takes (0..13, D = max_depth + 2 vertices at
most per walk), every min_depth, every pair of walk lengths and the camera
walk's emissive / background patterns that matter, the connections that
bdpt_pair_case lists must

* fit each case's list capacity per sample (bd_case_cap), so that a chunk's
  lists never overflow;
* map to distinct slots below D (D + 1) / 2 (bd_slot), the gather's mask
  width being 128 bits;
* be exactly the (s, t) pairs that sample_path's connection loop
  (bdpt_renderer.cpp:292-468) would run and could keep.
"""
from __future__ import annotations

import itertools

import pytest

S0, S1, T1, ST, NONE = 0, 1, 2, 3, 4


def pair_case(min_depth, max_depth, use_t1, emit, s, t):
    """bdpt_pair_case (bdpt.cuh): the case of connection (s, t), NONE when the
    loop skips it or always rejects it."""
    if t == 1 and not use_t1:
        return NONE
    if s + t < min_depth + 2 or s + t > max_depth + 2:
        return NONE
    bg = (emit >> (16 + t - 1)) & 1
    light = (emit >> (t - 1)) & 1
    if s > 0 and bg:
        return NONE
    if s == 0:
        return S0 if (bg or light) else NONE
    if t == 1:
        return T1
    return S1 if s == 1 else ST


def slot(D, s, t):
    """bd_slot (bdpt.cu): host-loop order, s outer, t inner."""
    return s * D - s * (s - 1) // 2 + t - 1


def case_cap(D, c):
    """bd_case_cap (bdpt.cu)."""
    return {S0: D - 1, S1: max(D - 2, 0), T1: D - 1}.get(c, (D - 3) * (D - 2) // 2 if D >= 4 else 0)


def emit_patterns(nt):
    """Camera-walk masks: no emitter, every vertex an area light, a
    background vertex last (it ends the walk), and both."""
    lights = (1 << nt) - 1
    bg_last = 1 << (16 + nt - 1) if nt else 0
    return [0, lights & ~1, bg_last, (lights & ~1) | bg_last]


@pytest.mark.parametrize("max_depth", range(14))
def test_lists_fit_and_slots_are_distinct(max_depth):
    D = max_depth + 2
    n_slots = D * (D + 1) // 2
    assert n_slots <= 128
    for min_depth, use_t1 in itertools.product(range(max_depth + 1), (True, False)):
        for ns in range(0, D + 1):
            for nt in range(1, D + 1):
                for emit in emit_patterns(nt):
                    counts = [0] * 4
                    slots = set()
                    for s in range(ns + 1):
                        for t in range(1, nt + 1):
                            c = pair_case(min_depth, max_depth, use_t1, emit, s, t)
                            if c == NONE:
                                continue
                            assert s + t <= D and s <= 15 and t <= 15
                            counts[c] += 1
                            if t >= 2:
                                k = slot(D, s, t)
                                assert 0 <= k < n_slots and k not in slots
                                slots.add(k)
                    for c in range(4):
                        assert counts[c] <= max(1, case_cap(D, c)), (max_depth, ns, nt, c)


def test_slots_follow_the_host_loop_order():
    """The gather sums a sample's slots in ascending order: that must be the
    host loop's (s outer, t inner) order, so the two add in the same order."""
    for D in range(2, 16):
        order = [slot(D, s, t) for s in range(D) for t in range(1, D - s + 1)]
        assert order == sorted(order) == list(range(D * (D + 1) // 2))


def test_listed_pairs_are_the_loop_pairs():
    """Against the connection loop's own branch ladder: every pair the loop
    would evaluate past its skips is listed, with the case of the branch it
    takes."""
    def loop_case(min_depth, max_depth, use_t1, emit, s, t):
        if t == 1 and not use_t1:
            return NONE
        if s + t < min_depth + 2 or s + t > max_depth + 2:
            return NONE
        bg = (emit >> (16 + t - 1)) & 1
        light = (emit >> (t - 1)) & 1
        if s > 0 and bg:
            return NONE
        if s == 1 and t == 1:
            return T1
        if s == 0 and t >= 2 and bg:
            return S0
        if s == 0 and t >= 2 and light:
            return S0
        if s == 0 and t >= 2:
            return NONE
        if s == 1 and t >= 2:
            return S1
        if s >= 2 and t == 1:
            return T1
        return ST
    for max_depth in (0, 1, 3, 8, 13):
        D = max_depth + 2
        for nt in range(1, D + 1):
            for emit in emit_patterns(nt):
                for s in range(D + 1):
                    for t in range(1, nt + 1):
                        for min_depth in (0, 1, max_depth):
                            for use_t1 in (True, False):
                                assert (pair_case(min_depth, max_depth, use_t1, emit, s, t) ==
                                        loop_case(min_depth, max_depth, use_t1, emit, s, t))
