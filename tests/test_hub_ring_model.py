"""A model of the hub targets' traversal (k_walk_f32_hubs in
grapher_b200/csrc/forces.cu): a warp takes ranges [lo, hi) of consecutive
sibling subtrees from a first-in first-out ring, tests each range's first
node, and appends the opened cell's children [lo + 1, min(next, hi)) and the
remaining siblings [next, hi) in lane order; a range that finds the ring full
is walked to its end by its lane. On random preorder trees with skip pointers
it must visit exactly the nodes the plain stackless walk visits (next node:
cur + 1 after an opened cell, else the skip pointer), each once, for any
ring size (no GPU)."""
import sys

import numpy as np
import pytest


def _random_preorder_tree(rng, n_nodes):
    """Preorder arrays of a random tree (<= 4 children a node): next[i] is
    the node after i's subtree, leaf[i] whether i has no children."""
    children = [[] for _ in range(n_nodes)]
    for v in range(1, n_nodes):
        while True:
            p = int(rng.integers(0, v))
            if len(children[p]) < 4:
                children[p].append(v)
                break
    order, nxt = [], {}

    def emit(v):
        order.append(v)
        for c in children[v]:
            emit(c)
        nxt[v] = len(order)

    sys.setrecursionlimit(max(sys.getrecursionlimit(), 4 * n_nodes))
    emit(0)
    next_ = np.array([nxt[order[i]] for i in range(n_nodes)])
    leaf = np.array([not children[order[i]] for i in range(n_nodes)])
    return next_, leaf


def _stackless(next_, leaf, opened, base, end):
    seen, cur = [], base
    while cur < end:
        seen.append(cur)
        cur = cur + 1 if (not leaf[cur] and opened[cur]) else max(next_[cur], cur + 1)
    return seen


def _ring(next_, leaf, opened, base, end, ring_size, take=2, lanes=32):
    seen = []
    ring = [None] * ring_size
    head, tail = 0, 0
    if base < end:
        ring[0], tail = (base, end), 1

    def serial(lo, hi):
        seen.extend(_stackless(next_, leaf, opened, lo, hi))

    while head < tail:
        n_take = min(tail - head, lanes * take)
        # lane l takes entries l, l + 32, ...; its outputs are appended in lane order
        per_lane = [[] for _ in range(lanes)]
        for u in range(take):
            for lane in range(lanes):
                k = lane + lanes * u
                if k >= n_take:
                    continue
                lo, hi = ring[(head + k) % ring_size]
                seen.append(lo)
                nxt = max(int(next_[lo]), lo + 1)
                is_open = (not leaf[lo]) and opened[lo]
                child_end = min(nxt, hi)
                if is_open and lo + 1 < child_end:
                    per_lane[lane].append((lo + 1, child_end))
                if nxt < hi:
                    per_lane[lane].append((nxt, hi))
        head += n_take
        room = ring_size - (tail - head)
        slot, appended = 0, 0
        for lane in range(lanes):
            for e in per_lane[lane]:
                if slot < room:
                    ring[(tail + slot) % ring_size] = e
                    appended += 1
                else:
                    serial(*e)
                slot += 1
        tail += appended
    return seen


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("ring_size", [4, 64, 1024])
def test_ring_visits_what_the_stackless_walk_visits(seed, ring_size):
    rng = np.random.default_rng(seed)
    next_, leaf = _random_preorder_tree(rng, 3000)
    opened = rng.random(3000) < 0.7           # the opening test's outcome per cell
    ref = _stackless(next_, leaf, opened, 0, 3000)
    got = _ring(next_, leaf, opened, 0, 3000, ring_size)
    assert len(got) == len(set(got))          # every node at most once
    assert sorted(got) == sorted(ref)


def test_everything_opened_visits_every_node():
    rng = np.random.default_rng(9)
    next_, leaf = _random_preorder_tree(rng, 2000)
    got = _ring(next_, leaf, np.ones(2000, bool), 0, 2000, 16)
    assert sorted(got) == list(range(2000))
