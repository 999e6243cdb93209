"""The treelet kernel's warp reductions restate two of the reference's loops in closed form
(optimizeTreelet, BVH/Optimization.cu:59-107 and :224-324).  These CPU tests check the
closed forms against the loops themselves on tie-heavy inputs:

* the partition bracket (for d = 16..1 lane l takes lane min(l+d, 31)'s candidate when its
  own is the empty -1 or the other is smaller) leaves in lane 0 the smallest cost, ties
  going to the lane whose 5-bit index read backwards is smallest, the empty candidate
  losing to any other;
* the formation scan (the first of lanes 0..size-1 whose area is the largest above -1, lane
  0 when none) picks the lowest lane holding the largest area bit pattern.
"""
import random


def bracket(tc, p):
    tc, p = list(tc), list(p)
    for d in (16, 8, 4, 2, 1):
        ntc, np_ = tc[:], p[:]
        for lane in range(32):
            o = min(lane + d, 31)
            if tc[lane] == -1.0 or tc[o] < tc[lane]:
                ntc[lane], np_[lane] = tc[o], p[o]
        tc, p = ntc, np_
    return tc[0], p[0]


def bitrev5(x: int) -> int:
    return int(f"{x:05b}"[::-1], 2)


def closed_form(tc, p):
    key = [float("inf") if v == -1.0 else v for v in tc]
    best = min(key)
    win = min((lane for lane in range(32) if key[lane] == best), key=bitrev5)
    return tc[win], p[win]


def test_partition_bracket_is_min_with_bit_reversed_ties():
    rng = random.Random(7)
    for _ in range(20_000):
        tc = [rng.choice([0.0, 0.5, 1.0, 1.5, 2.0, 3.0]) for _ in range(32)]
        if rng.random() < 0.5:
            tc[0] = -1.0  # the 6-leaf stage: lane 0 has no partition
        p = [rng.randrange(1, 128) for _ in range(32)]
        assert bracket(tc, p) == closed_form(tc, p)


def test_seven_leaf_prestep_then_bracket():
    # the 7-leaf stage: lane l holds partitions l and l | 32 and keeps the smaller (lane 0's
    # first one is empty), then the same bracket
    rng = random.Random(11)
    for _ in range(5_000):
        c = [rng.choice([1.0, 2.0, 2.5]) for _ in range(64)]
        tc, p = [], []
        for lane in range(32):
            t, q = (-1.0 if lane == 0 else c[lane]), lane
            if t == -1.0 or c[lane | 32] < t:
                t, q = c[lane | 32], lane | 32
            tc.append(t)
            p.append(q)
        assert bracket(tc, p) == closed_form(tc, p)


def test_formation_scan_is_first_lane_with_largest_area():
    import struct

    def bits(x: float) -> int:
        return struct.unpack("<I", struct.pack("<f", x + 0.0))[0]

    rng = random.Random(13)
    for _ in range(20_000):
        size = rng.choice([1, 3, 5, 7, 9, 11])
        area = [rng.choice([0.0, 0.25, 1.0, 4.0, float("inf")]) for _ in range(32)]
        eligible = [lane < size and rng.random() < 0.7 for lane in range(32)]
        # the reference's scan
        my = [area[i] if eligible[i] else -1.0 for i in range(32)]
        max_lane, max_area = 0, -1.0
        for i in range(size):
            if my[i] > max_area:
                max_area, max_lane = my[i], i
        # the reduction: key = area bits + 1 for candidates, 0 otherwise; first lane of the max
        key = [bits(area[i]) + 1 if (eligible[i] and area[i] > -1.0) else 0 for i in range(32)]
        top = max(key)
        fast = key.index(top) if top != 0 else 0
        assert fast == max_lane
