"""The slice-order rule of the sliced-ELL layout in 2D (lpm-cpp_b200/csrc/topology.cu: spread_slices),
restated and checked on slice-width profiles like those of the lattice generators.

After the row sort (descending connection count), a problem's narrow slices (boundary particles) sit
at the end of its slice order, so a split of the slices into equal-cost ranges (the batched CG's
split, batch.cu: batch_split) gives them all to the last blocks.  The rule reorders whole slices:
slice s of width class c and rank r within the class gets key (r + 1/2) / |c|; slices are ordered by
(key, width descending, old position).  A partial last slice (n not a multiple of 32) stays last.

Invariants checked: the order is a permutation that keeps a partial last slice last; within each
width class the old order is kept; every width class is spread (any prefix of the new order holds
its proportional share of each class within as many slices as there are classes); and equal-slot
ranges of the new order hold about equal shares of narrow slices, which the old order does not."""
import numpy as np
import pytest


def spread_order(widths, n):
    """The reordering of topology.cu: returns the new slice order as old slice indices."""
    nslices = len(widths)
    nmove = nslices if n % 32 == 0 else nslices - 1
    if nmove < 2:
        return list(range(nslices))
    count, seen, keys = {}, {}, []
    for w in widths[:nmove]:
        count[w] = count.get(w, 0) + 1
    for s in range(nmove):
        w = widths[s]
        keys.append(((seen.get(w, 0) + 0.5) / count[w], -w, s))
        seen[w] = seen.get(w, 0) + 1
    order = [k[2] for k in sorted(keys)]
    return order + list(range(nmove, nslices))


def plate_widths(rng, nslices, interior=31, narrow_frac=0.12, classes=None):
    """Descending-count slice widths: interior slices at full width, then narrower boundary ones
    (widths drawn from `classes`, or from 12..interior-1)."""
    nb = max(1, int(nslices * narrow_frac))
    pool = np.arange(12, interior) if classes is None else np.asarray(classes)
    tail = np.sort(rng.choice(pool, size=nb))[::-1]
    return [interior] * (nslices - nb) + [int(x) for x in tail]


@pytest.mark.parametrize("seed", range(6))
def test_spread_is_a_class_preserving_permutation(seed):
    rng = np.random.default_rng(seed)
    nslices = int(rng.integers(20, 900))
    n = nslices * 32 - int(rng.integers(0, 32))
    w = plate_widths(rng, nslices)
    order = spread_order(w, n)
    assert sorted(order) == list(range(nslices))
    if n % 32:
        assert order[-1] == nslices - 1
    # within a width class the old order is kept
    for c in set(w):
        pos = [order.index(s) for s in range(nslices) if w[s] == c]
        assert pos == sorted(pos)


@pytest.mark.parametrize("seed", range(6))
def test_each_width_class_is_spread_evenly(seed):
    rng = np.random.default_rng(100 + seed)
    nslices = int(rng.integers(64, 900))
    n = nslices * 32
    w = plate_widths(rng, nslices, narrow_frac=float(rng.uniform(0.05, 0.3)))
    order = spread_order(w, n)
    neww = np.array([w[s] for s in order])
    for c in set(w):
        ind = (neww == c).astype(float)
        share = ind.mean()
        cum = np.concatenate([[0.0], np.cumsum(ind)])
        # a prefix of the new order ends at some key value v: each class contributes the slices
        # whose keys are below v, within one of its proportional share, so class c's count is off
        # by at most one plus the other classes' rounding (one each)
        dev = np.abs(cum - share * np.arange(len(cum)))
        assert dev.max() <= len(set(w)), (c, dev.max())


def test_equal_cost_ranges_get_equal_narrow_shares():
    # a lattice's boundary rows come in a few connection counts, each class with many slices
    rng = np.random.default_rng(7)
    nslices, G = 640, 24
    w = plate_widths(rng, nslices, narrow_frac=0.15, classes=(27, 23, 19))
    def narrow_per_range(order):
        widths = np.array([w[s] for s in order])
        cum = np.concatenate([[0], np.cumsum(widths)])
        bounds = np.searchsorted(cum, np.arange(G + 1) * cum[-1] / G)
        return np.array([(widths[bounds[b]:bounds[b + 1]] < 31).sum() for b in range(G)])
    before = narrow_per_range(list(range(nslices)))
    after = narrow_per_range(spread_order(w, nslices * 32))
    # the sorted order puts every narrow slice in the last few ranges; the spread order gives each
    # range about the same number
    assert before[: G // 2].sum() == 0 and before.max() > 3 * after.max()
    assert after.max() <= 2 * after.mean() and after.min() >= after.mean() / 2, after
