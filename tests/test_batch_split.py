"""The integer rules of the batched CG's split (lpm-cpp_b200/csrc/batch.cu: seg_block, seg_bound,
slice_at, batch_split), restated and checked on random mixes of problem sizes.  The active
problems' costs are laid end to end and cut into G equal segments, one per block; a problem's
piece in a block is its part of that segment, rounded to whole slices by their starting cost.

Invariants: the pieces of each problem cover its slices exactly once and in order; pieces are
numbered contiguously per problem (partial slots); no block carries more than its equal share
plus one slice; and the total piece count stays within G + problems - 1 (the partial buffers)."""
import numpy as np
import pytest


def seg_block(t, C, G):
    b = ((t + 1) * G + C - 1) // C - 1
    return min(b, G - 1)


def seg_bound(b, C, G):
    return b * C // G


def slice_at(slice_off, v):
    # first s with slice_off[s] >= v
    return int(np.searchsorted(slice_off, v, side="left"))


def split(problems, G):
    """problems: list of (slice_off array, dim).  Returns per block its pieces
    [(rank, s0, s1, slot)] and the slot count, as every block of the kernel computes them."""
    costs = [int(so[-1]) * (d * d + 1) for so, d in problems]
    cum = np.concatenate([[0], np.cumsum(costs)]).astype(np.int64)
    C = int(cum[-1])
    fb = [seg_block(int(cum[r]), C, G) for r in range(len(problems))]
    lb = [seg_block(int(cum[r + 1]) - 1, C, G) for r in range(len(problems))]
    g = [l - f + 1 for f, l in zip(fb, lb)]
    vs = np.concatenate([[0], np.cumsum(g)])[:-1]
    blocks = []
    for b in range(G):
        pieces = []
        for r, (so, d) in enumerate(problems):
            if not (fb[r] <= b <= lb[r]):
                continue
            c0, c1 = int(cum[r]), int(cum[r + 1])
            lo = max(seg_bound(b, C, G), c0) - c0
            hi = max(lo, min(seg_bound(b + 1, C, G), c1) - c0)
            e1 = d * d + 1
            pieces.append((r, slice_at(so, -(-lo // e1)), slice_at(so, -(-hi // e1)), int(vs[r]) + b - fb[r]))
        blocks.append(pieces)
    return blocks, int(sum(g)), C


def random_problems(rng, count):
    out = []
    for _ in range(count):
        ns = int(rng.integers(1, 400))
        widths = np.sort(rng.integers(1, 62, ns))[::-1]  # sliced-ELL rows sorted by width
        out.append((np.concatenate([[0], np.cumsum(widths)]).astype(np.int64), int(rng.choice([2, 3]))))
    return out


@pytest.mark.parametrize("G", [1, 7, 148, 1000])
@pytest.mark.parametrize("seed", range(6))
def test_split_partitions_every_problem(G, seed):
    rng = np.random.default_rng(seed)
    problems = random_problems(rng, int(rng.integers(1, 65)))
    blocks, nslots, C = split(problems, G)
    assert nslots <= G + len(problems) - 1
    covered = {r: [] for r in range(len(problems))}
    slots = {r: [] for r in range(len(problems))}
    for b, pieces in enumerate(blocks):
        for r, s0, s1, slot in pieces:
            covered[r].append((s0, s1))
            slots[r].append(slot)
        # one block's matrix volume: its equal share plus at most one slice of rounding
        vol = sum((problems[r][0][s1] - problems[r][0][s0]) * (problems[r][1] ** 2 + 1) for r, s0, s1, _ in pieces)
        max_slice = max(int(np.diff(so).max()) * (d * d + 1) for so, d in problems)
        assert vol <= C // G + 2 * max_slice + 1
    for r, (so, _) in enumerate(problems):
        ranges = covered[r]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(so) - 1
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:])), "pieces must be contiguous and in order"
        assert all(s0 <= s1 for s0, s1 in ranges)
        assert slots[r] == list(range(slots[r][0], slots[r][0] + len(slots[r]))), "contiguous partial slots"
    all_slots = sorted(s for v in slots.values() for s in v)
    assert all_slots == list(range(nslots)), "every partial slot is written by exactly one piece"


def test_split_balances_the_64_plate_mix():
    """Sizes like the 64-plate workload (460 to 18,000 particles): every SM gets work and the
    largest block carries at most a few percent over the equal share, where giving each problem one
    block plus a share of the rest left 28 SMs idle and loaded the busiest 1.75x."""
    rng = np.random.default_rng(20240604)
    problems = []
    for _ in range(64):
        side = float(np.exp(rng.uniform(np.log(4.0), np.log(25.0))))
        n = int(29 * side * side)
        ns = -(-n // 32)
        widths = np.full(ns, 30)
        problems.append((np.concatenate([[0], np.cumsum(widths)]).astype(np.int64), 2))
    blocks, _, C = split(problems, 148)
    vols = [sum((problems[r][0][s1] - problems[r][0][s0]) * 5 for r, s0, s1, _ in p) for p in blocks]
    assert min(vols) > 0
    assert max(vols) <= 1.05 * C / 148
