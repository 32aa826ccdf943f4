"""The persistent stage 2's task order (decode() in soi_fft_b200/csrc/stage2_fast.cuh),
restated here to check the properties its deadlock-freedom argument rests on:
every (pass, segment, tile) is claimed exactly once, a segment's pass-2 tasks come
after all of its pass-1 tasks (a pass-2 task only waits on smaller claim indices),
and from the second segment on at least `tail` claims separate a segment's last
pass-1 task from its first pass-2 task.  With tail = NT2 the order is the
original one: every pass-1 task of a block before its pass-2 tasks.
(tests/test_gpu_segments.py checks on the GPU that the order does not change
results.)"""
import pytest


def decode(t, nt1, nt2, S, tail):
    per = nt1 + nt2
    if t < nt1:
        return (1, 0, t)
    blk, r = divmod(t - nt1, per)
    if blk >= S - 1:
        return (2, blk, r)
    n2i = nt2 - tail
    ni = nt1 + n2i
    if r >= ni:
        return (2, blk, n2i + (r - ni))
    c0, c1 = r * nt1 // ni, (r + 1) * nt1 // ni
    return (1, blk + 1, c0) if c1 > c0 else (2, blk, r - c0)


def decode_all_pass1_first(t, nt1, nt2, S):
    per = nt1 + nt2
    if t < nt1:
        return (1, 0, t)
    blk, r = divmod(t - nt1, per)
    if blk < S - 1 and r < nt1:
        return (1, blk + 1, r)
    return (2, blk, r - (nt1 if blk < S - 1 else 0))


@pytest.mark.parametrize("nt1,nt2,S", [(512, 640, 128), (128, 320, 32), (64, 80, 16), (512, 512, 3),
                                       (64, 80, 1), (8, 5, 4), (1024, 1280, 8)])
def test_claim_order_is_complete_and_ordered(nt1, nt2, S):
    total = S * (nt1 + nt2)
    for tail in sorted({0, 1, min(296, nt2), nt2 // 2, nt2}):
        seen, last_p1, first_p2 = set(), {}, {}
        for t in range(total):
            k = decode(t, nt1, nt2, S, tail)
            assert k not in seen
            seen.add(k)
            kind, seg, tile = k
            assert 0 <= seg < S and 0 <= tile < (nt1 if kind == 1 else nt2)
            if kind == 1:
                last_p1[seg] = t
            else:
                first_p2.setdefault(seg, t)
            if tail == nt2:
                assert k == decode_all_pass1_first(t, nt1, nt2, S)
        assert len(seen) == total
        for seg in range(S):
            assert first_p2[seg] > last_p1[seg]
            if seg > 0:
                assert first_p2[seg] - last_p1[seg] >= tail + 1
