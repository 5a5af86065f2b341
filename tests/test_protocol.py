"""CPU model of the reduction's lock-free protocol, checked against the oracle.

The GPU reduces columns concurrently: a column adds the published version of
its lowest row's current owner (a snapshot that may be stale), claims the row
when it has no owner or a larger one (displacing that owner, which then goes
on from its own published version), clears the claimed row's column (twist),
and stops as zero once its own column has been cleared, even in the middle of
a reduction or before the higher dimension is finished.  This model
interleaves single additions of all columns in a random order, dimensions
mixed, and checks that every schedule ends with the oracle's pairs and
essential classes: the order independence the concurrent tiers and the
dimension gate rely on."""
import numpy as np
import pytest

import oracle
from helpers import random_complex


def simulate(m, rng, clear=True):
    n = m.ncols
    work = [set(int(x) for x in m.column(j)) for j in range(n)]
    pub = {}      # owner column -> its published version (immutable snapshot)
    owner = {}    # row -> owner column
    cleared = set()
    active = [j for j in range(n) if work[j]]
    zero = set(j for j in range(n) if not work[j])
    while active:
        k = int(rng.integers(len(active)))
        j = active[k]
        if clear and j in cleared:  # positive: stops as zero
            active[k] = active[-1]
            active.pop()
            zero.add(j)
            continue
        w = work[j]
        if not w:
            active[k] = active[-1]
            active.pop()
            zero.add(j)
            continue
        r = max(w)
        o = owner.get(r)
        if o is not None and o < j:  # one addition, then any column may move next
            w ^= pub[o]
            continue
        owner[r] = j  # claim (displacing a larger owner)
        pub[j] = frozenset(w)
        active[k] = active[-1]
        active.pop()
        if clear:
            cleared.add(r)
        if o is not None:
            active.append(o)  # displaced: goes on from its published version
    pairs = np.array(sorted(owner.items()), dtype=np.int64).reshape(-1, 2)
    owned = set(owner)
    ess = np.array(sorted(j for j in zero if j not in owned), dtype=np.int64)
    return pairs, ess


@pytest.mark.parametrize("seed", range(12))
def test_every_schedule_gives_the_oracle_pairs(seed):
    rng = np.random.default_rng(4400 + seed)
    m = random_complex(rng, nverts=int(rng.integers(6, 11)), p=float(rng.uniform(0.4, 0.8)), maxdim=3)
    ref = oracle.reduce(m)
    for trial in range(6):
        pairs, ess = simulate(m, np.random.default_rng(seed * 100 + trial), clear=trial % 3 != 2)
        assert np.array_equal(pairs, ref.pairs), trial
        assert np.array_equal(ess, ref.essential), trial
