"""The identities the GPU octree build relies on, checked on the CPU.

The build (n_body_sim_pro_b200/csrc/bh.cu) is a Karras radix tree over the
sorted Morton keys (ties broken by index), then an octree of buckets:

* radix_tree_kernel decides whether a binary node is an octree cell from its
  own range: the parent's common-prefix length is that of the node's range
  extended by one key on the side with the longer common prefix,
  max(delta(first - 1, first), delta(last, last + 1));
* keep_kernel / place_kernel take the octree children of a splitting cell (an
  octree cell of more than `leaf_capacity` particles above level 21) as the
  first cells below it in the binary tree, and keep exactly those cells and
  the root.

Here a plain-Python restatement of the radix tree (small random key sets with
repeated keys and clustered prefixes) checks both against the explicit
definitions: the parent read from the built tree, and the octree parent found
by climbing the binary tree (the cell kept when its octree parent has more
than `leaf_capacity` particles).
"""
import random

import pytest


def _clz64(x):
    return 64 - x.bit_length()


def _clz32(x):
    return 32 - x.bit_length()


def _prefix(keys, i, j):
    """Common prefix length of sorted keys i and j in bits; the index breaks
    ties between equal keys; -1 outside the array (bh.cu prefix())."""
    n = len(keys)
    if j < 0 or j >= n:
        return -1
    a, b = keys[i], keys[j]
    if a != b:
        return _clz64(a ^ b) - 1  # 63-bit keys
    return 63 + _clz32(i ^ j)


def _level(delta):
    # C integer division truncates towards zero: delta = -1 gives level 0
    return min(int(delta / 3), 21)


def _radix_tree(keys):
    """Karras (2012): range, split children and prefix length of every internal
    node; binary ids: internal i -> i, particle k -> (n - 1) + k."""
    n = len(keys)
    rng, child, delta = [None] * (n - 1), [None] * (n - 1), [0] * (n - 1)
    parent = [-1] * (2 * n - 1)
    for i in range(n - 1):
        d = 1 if _prefix(keys, i, i + 1) - _prefix(keys, i, i - 1) >= 0 else -1
        dmin = _prefix(keys, i, i - d)
        lmax = 2
        while _prefix(keys, i, i + lmax * d) > dmin:
            lmax <<= 1
        length, step = 0, lmax >> 1
        while step >= 1:
            if _prefix(keys, i, i + (length + step) * d) > dmin:
                length += step
            step >>= 1
        j = i + length * d
        dnode = _prefix(keys, i, j)
        s, div = 0, 2
        while True:
            step = (length + div - 1) // div
            if _prefix(keys, i, i + (s + step) * d) > dnode:
                s += step
            if step <= 1:
                break
            div <<= 1
        gamma = i + s * d + (-1 if d < 0 else 0)
        first, last = min(i, j), max(i, j)
        left = (n - 1) + gamma if first == gamma else gamma
        right = (n - 1) + gamma + 1 if last == gamma + 1 else gamma + 1
        rng[i], child[i], delta[i] = (first, last), (left, right), dnode
        parent[left] = parent[right] = i
    return rng, child, delta, parent


def _cells_from_parents(n, delta, parent):
    """Octree cell level of every binary node from its parent's prefix length
    (the definition; -1: not a cell, 22: a particle in a cell of its own)."""
    cell = [-1] * (2 * n - 1)
    for b in range(2 * n - 1):
        p = parent[b]
        if b < n - 1:
            lvl = _level(delta[b])
            if b == 0 or _level(delta[p]) < lvl:
                cell[b] = lvl
        elif _level(delta[p]) <= 20:
            cell[b] = 22
    return cell


def _cells_from_ranges(keys, rng, child, delta):
    """The same from each node's own range, as radix_tree_kernel decides it."""
    n = len(keys)
    cell = [None] * (2 * n - 1)
    for i in range(n - 1):
        first, last = rng[i]
        lvl = _level(delta[i])
        pdelta = max(_prefix(keys, first, first - 1), _prefix(keys, last, last + 1))
        cell[i] = lvl if (i == 0 or _level(pdelta) < lvl) else -1
        for c in child[i]:
            if c >= n - 1:
                cell[c] = 22 if lvl <= 20 else -1
    return cell


def _count(n, rng, b):
    return 1 if b >= n - 1 else rng[b][1] - rng[b][0] + 1


def _kept_by_climbing(n, rng, parent, cell, cap):
    """A cell is kept when its octree parent (the nearest binary ancestor that
    is a cell) has more than `cap` particles; the root always is."""
    kept = {0: -1}
    for b in range(1, 2 * n - 1):
        if cell[b] < 0:
            continue
        p = parent[b]
        while cell[p] < 0:
            p = parent[p]
        if _count(n, rng, p) > cap:
            kept[b] = p
    return kept


def _kept_by_descent(n, rng, child, cell, cap):
    """keep_kernel: each splitting cell finds its octree children by descending
    the binary nodes of its own level; the root is kept."""
    def splits(b):
        return b < n - 1 and 0 <= cell[b] < 21 and _count(n, rng, b) > cap

    kept = {0: -1}
    for b in range(n - 1):
        if not splits(b):
            continue
        stack, kids = [child[b][1], child[b][0]], []
        while stack:
            c = stack.pop()
            if cell[c] >= 0:
                kids.append(c)
            else:
                assert c < n - 1, "a particle that is no cell below a splitting cell"
                stack += [child[c][1], child[c][0]]
        assert 1 <= len(kids) <= 8
        firsts = [rng[c][0] if c < n - 1 else c - (n - 1) for c in kids]
        assert firsts == sorted(firsts), "children in Morton (depth-first) order"
        for c in kids:
            kept[c] = b
    return kept


def _random_keys(rnd, n):
    """Sorted 63-bit keys: clustered prefixes (few top digits), some runs of
    equal keys (index tie-breaks), some all-distinct low bits."""
    keys = []
    for _ in range(n):
        top = rnd.choice([0, 1, 5, 7]) << 60
        mid = rnd.getrandbits(rnd.choice([3, 9, 30])) << 27
        low = rnd.getrandbits(27) if rnd.random() < 0.8 else 0
        keys.append((top | mid | low) & ((1 << 63) - 1))
    if n > 4:
        for _ in range(rnd.randint(0, 3)):  # duplicated keys
            k = rnd.randrange(n)
            keys[rnd.randrange(n)] = keys[k]
    return sorted(keys)


@pytest.mark.parametrize("seed", range(12))
def test_cell_levels_from_ranges_equal_the_parent_definition(seed):
    rnd = random.Random(seed)
    for _ in range(20):
        keys = _random_keys(rnd, rnd.randint(2, 160))
        rng, child, delta, parent = _radix_tree(keys)
        assert _cells_from_ranges(keys, rng, child, delta) == \
            _cells_from_parents(len(keys), delta, parent)


@pytest.mark.parametrize("cap", [1, 2, 4, 16])
def test_kept_cells_by_descent_equal_the_climbing_definition(cap):
    rnd = random.Random(100 + cap)
    for _ in range(40):
        keys = _random_keys(rnd, rnd.randint(2, 200))
        n = len(keys)
        rng, child, delta, parent = _radix_tree(keys)
        cell = _cells_from_ranges(keys, rng, child, delta)
        assert _kept_by_descent(n, rng, child, cell, cap) == \
            _kept_by_climbing(n, rng, parent, cell, cap)
