"""Order of the keys visited by a T1 sweep, on a model of its two queues (host only).

A sweep visits the sorted candidate keys in ascending order, and every flip queues the keys of the
short edges it moved or rewired (each greater than the key being visited), which are visited in
their place. The reference's CPU sweep keeps one sorted list. The device sweep keeps the candidates
in a sorted array and the queued keys in a binary min-heap; a key queued more than once is popped
with all its copies, and a queued key that is also a candidate is visited once. This test checks,
on random candidate lists and random queued keys, that both visit the same keys in the same order.
The heap follows the device code's push and pop (cellgpu_b200/csrc/vertex.cu: heap_push,
heap_pop, heap_pop_unique).
"""
import numpy as np
import pytest


def heap_push(h, key):
    h.append(key)
    i = len(h) - 1
    while i > 0:
        p = (i - 1) >> 1
        if h[p] <= key:
            break
        h[i] = h[p]
        i = p
    h[i] = key


def heap_pop(h):
    top = h[0]
    last = h.pop()
    n = len(h)
    if n == 0:
        return top
    i = 0
    while True:
        l = 2 * i + 1
        if l >= n:
            break
        c = l + 1 if l + 1 < n and h[l + 1] < h[l] else l
        if last <= h[c]:
            break
        h[i] = h[c]
        i = c
    h[i] = last
    return top


def sweep_sorted_queue(cands, queued_by):
    """One sorted queue; a queued key is inserted into the pending part unless already there."""
    q = sorted(cands)
    head, order = 0, []
    while head < len(q):
        key = q[head]
        head += 1
        order.append(key)
        for k2 in queued_by(key):
            if k2 <= key:
                continue
            pending = q[head:]
            if k2 in pending:
                continue
            pos = head + int(np.searchsorted(pending, k2))
            q.insert(pos, k2)
    return order


def sweep_heap(cands, queued_by):
    """Sorted candidates and a min-heap of queued keys, merged in ascending order."""
    main = sorted(cands)
    h, hm, order = [], 0, []
    while hm < len(main) or h:
        if h and (hm >= len(main) or h[0] <= main[hm]):
            key = heap_pop(h)
            while h and h[0] == key:
                heap_pop(h)
            if hm < len(main) and main[hm] == key:
                hm += 1
        else:
            key = main[hm]
            hm += 1
        order.append(key)
        for k2 in queued_by(key):
            if k2 > key:
                heap_push(h, k2)
    return order


@pytest.mark.parametrize("seed", range(40))
def test_heap_sweep_visits_the_sorted_queue_order(seed):
    rng = np.random.default_rng(seed)
    n_keys = int(rng.integers(1, 400))
    universe = 3 * n_keys
    cands = sorted(set(rng.integers(0, universe, size=n_keys).tolist()))
    p_flip = rng.uniform(0.0, 0.8)
    table = {}

    def queued_by(key):
        # a fixed set of keys per visited key (duplicates and keys already queued included), as
        # a flip's twelve rewired edges can name a key twice or one that is still pending
        if key not in table:
            r = np.random.default_rng(seed * 100003 + key)
            if r.random() < p_flip:
                # keys are edge keys of the instance: below 3 x its vertex count
                ks = [k for k in r.integers(key - 3, key + 40, size=int(r.integers(1, 13))).tolist()
                      if k < universe]
                ks += ks[: int(r.integers(0, 3))]
            else:
                ks = []
            table[key] = ks
        return table[key]

    assert sweep_heap(cands, queued_by) == sweep_sorted_queue(cands, queued_by)
