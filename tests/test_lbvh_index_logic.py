"""CPU restatement of the index logic of the device BVH build (sol_b200/csrc/kernels/lbvh.cu).

The device build cannot run here, and its failures would be out-of-range
accesses on the GPU, so its integer logic is restated step for step and
checked on random inputs: the radix tree over sorted 63-bit keys with the
position tie-break (Karras, HPG 2012), the bottom-up SAH costs and leaf
decisions, the 7-leaf treelet restructuring by subset dynamic programming
(Karras and Aila, HPG 2013), the depth-first triangle positions and the rule
for which internal nodes are emitted.  Checked: a valid binary tree
(parents and children agree, every triangle under exactly one leaf), counts
and boxes consistent after rewiring, leaves covering consecutive positions,
emitted nodes exactly those reachable from the root, and an SAH cost that
never rises from pass to pass.  The GPU tests check the device build itself
(tests/test_gpu_lbvh.py)."""
import random

import pytest

LEAF_MAX = 8
TREELET = 7


def clz64(x):
    return 64 - x.bit_length()


def clz32(x):
    return 32 - x.bit_length()


def half_area(b):
    dx, dy, dz = b[3] - b[0], b[4] - b[1], b[5] - b[2]
    return dx * dy + dy * dz + dz * dx


def union(a, b):
    return [min(a[0], b[0]), min(a[1], b[1]), min(a[2], b[2]), max(a[3], b[3]), max(a[4], b[4]), max(a[5], b[5])]


def radix_tree(keys):
    """radix_tree: children (>= 0 internal, < 0 ~sorted triangle), parents, counts."""
    n = len(keys)

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        x = keys[i] ^ keys[j]
        return clz64(x) if x else 64 + clz32(i ^ j)

    child, parent_i, parent_l, count = [None] * (n - 1), [None] * (n - 1), [None] * n, [0] * (n - 1)
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) > 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax *= 2
        l, t = 0, lmax // 2
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t //= 2
        j = i + l * d
        assert 0 <= j < n and l >= 1
        dnode = delta(i, j)
        s, div = 0, 2
        t = (l + div - 1) // div
        while True:
            if delta(i, i + (s + t) * d) > dnode:
                s += t
            if t == 1:
                break
            div *= 2
            t = (l + div - 1) // div
        gamma = i + s * d + min(d, 0)
        first, last = min(i, j), max(i, j)
        assert first <= gamma < last
        count[i] = last - first + 1
        left = ~gamma if first == gamma else gamma
        right = ~(gamma + 1) if last == gamma + 1 else gamma + 1
        child[i] = [left, right]
        for c in (left, right):
            if c >= 0:
                assert parent_i[c] is None
                parent_i[c] = i
            else:
                assert parent_l[~c] is None
                parent_l[~c] = i
    return child, parent_i, parent_l, count


class Tree:
    def __init__(self, tri_boxes, keys):
        self.tb = tri_boxes
        self.child, self.pi, self.pl, self.count = radix_tree(keys)
        m = len(keys) - 1
        self.box, self.cost, self.leaf = [None] * m, [0.0] * m, [0] * m

    def info(self, ref):
        if ref >= 0:
            return self.box[ref], self.cost[ref], self.count[ref]
        b = self.tb[~ref]
        return b, half_area(b), 1

    def set_parent(self, ref, parent):
        if ref >= 0:
            self.pi[ref] = parent
        else:
            self.pl[~ref] = parent


def restructure(t, root):
    """restructure: grow the treelet, subset DP, rewire when cheaper."""
    c0 = t.child[root]
    leaf = [c0[0], c0[1]]
    info = [t.info(leaf[0]), t.info(leaf[1])]
    inner = [root]
    while len(leaf) < TREELET:
        best, best_area = -1, -1.0
        for k, ref in enumerate(leaf):
            if ref >= 0 and half_area(info[k][0]) > best_area:
                best, best_area = k, half_area(info[k][0])
        if best < 0:
            break
        node = leaf[best]
        cc = t.child[node]
        inner.append(node)
        leaf[best], info[best] = cc[0], t.info(cc[0])
        leaf.append(cc[1])
        info.append(t.info(cc[1]))
    nl = len(leaf)
    if nl < 3:
        return
    full = (1 << nl) - 1
    cost, cnt, part = [0.0] * (full + 1), [0] * (full + 1), [0] * (full + 1)
    for s in range(1, full + 1):
        if s & (s - 1) == 0:
            k = (s & -s).bit_length() - 1
            cost[s], cnt[s] = info[k][1], info[k][2]
            continue
        b, n = None, 0
        for k in range(nl):
            if s >> k & 1:
                b = info[k][0] if b is None else union(b, info[k][0])
                n += info[k][2]
        a, low = half_area(b), s & -s
        best, bp = 3.0e38, low
        p = (s - 1) & s
        while p:
            if p & low and cost[p] + cost[s ^ p] < best:
                best, bp = cost[p] + cost[s ^ p], p
            p = (p - 1) & s
        split, as_leaf = a + best, n * a
        make_leaf = n <= LEAF_MAX and not (s == full and root == 0) and as_leaf <= split
        cnt[s], cost[s], part[s] = n, (as_leaf if make_leaf else split), bp | (0x80 if make_leaf else 0)
    if not cost[full] < t.cost[root] * 0.999999:
        return
    made, nxt, stack = [], 1, [(full, root)]
    while stack:
        s, node = stack.pop()
        made.append((s, node))
        l = part[s] & 0x7F
        refs = []
        for side in (l, s ^ l):
            if side & (side - 1) == 0:
                ref = leaf[(side & -side).bit_length() - 1]
            else:
                ref = inner[nxt]
                nxt += 1
                stack.append((side, ref))
            t.set_parent(ref, node)
            refs.append(ref)
        t.child[node] = refs
    assert nxt == len(inner)   # the treelet's own internal nodes, each reused once
    for s, node in made:
        b = None
        for k in range(nl):
            if s >> k & 1:
                b = info[k][0] if b is None else union(b, info[k][0])
        t.box[node], t.count[node], t.cost[node] = b, cnt[s], cost[s]
        t.leaf[node] = 1 if part[s] & 0x80 else 0


def bottom_up(t, node):
    """One pass of bottom_up, in an order where every node follows its children."""
    for c in list(t.child[node]):
        if c >= 0:
            bottom_up(t, c)
    a, b = t.info(t.child[node][0]), t.info(t.child[node][1])
    box = union(a[0], b[0])
    area, count = half_area(box), a[2] + b[2]
    split, as_leaf = area + a[1] + b[1], count * area
    leaf = node != 0 and count <= LEAF_MAX and as_leaf <= split
    t.box[node], t.count[node] = box, count
    t.cost[node], t.leaf[node] = (as_leaf if leaf else split), (1 if leaf else 0)
    if count > LEAF_MAX:
        restructure(t, node)


def first_position(t, ref):
    pos, node = 0, ref
    p = (t.pi[ref] if ref != 0 else -1) if ref >= 0 else t.pl[~ref]
    while p >= 0:
        c = t.child[p]
        if c[1] == node:
            pos += t.count[c[0]] if c[0] >= 0 else 1
        node, p = p, (-1 if p == 0 else t.pi[p])
    return pos


def emitted(t, i):
    if i == 0:
        return True
    if t.leaf[i]:
        return False
    p, guard = t.pi[i], 0
    while p != 0:
        if t.leaf[p]:
            return False
        if t.count[p] > LEAF_MAX:
            break
        p, guard = t.pi[p], guard + 1
        assert guard < 16
    return True


def build_and_check(n, seed, duplicate_keys):
    rnd = random.Random(seed)
    boxes = []
    for i in range(n):
        cx, cy, cz = (rnd.random() * 10 for _ in range(3))
        s = rnd.random() ** 3 * (5 if i % 50 == 0 else 0.2)
        boxes.append([cx - s, cy - s * 0.5, cz - s * 0.3, cx + s, cy + s * 0.7, cz + s])
    codes = [rnd.getrandbits(3) if duplicate_keys else rnd.getrandbits(63) for _ in range(n)]
    order = sorted(range(n), key=lambda j: (codes[j], j))   # a stable sort of (code, index) pairs
    t = Tree([boxes[j] for j in order], [codes[j] for j in order])
    sah = []
    for _ in range(3):
        bottom_up(t, 0)
        sah.append(t.cost[0] / half_area(t.box[0]))
    # A valid binary tree with parents and children in agreement.
    seen, tris, stack = set(), [], [0]
    while stack:
        i = stack.pop()
        assert i not in seen
        seen.add(i)
        for c in t.child[i]:
            if c >= 0:
                assert t.pi[c] == i
                stack.append(c)
            else:
                assert t.pl[~c] == i
                tris.append(~c)
    assert len(seen) == n - 1 and sorted(tris) == list(range(n))

    def check(i):
        total, box = 0, None
        for c in t.child[i]:
            cn, cb = check(c) if c >= 0 else (1, t.tb[~c])
            total, box = total + cn, (cb if box is None else union(box, cb))
        assert total == t.count[i] and box == t.box[i]
        return total, box
    check(0)
    pos = [first_position(t, ~j) for j in range(n)]
    assert sorted(pos) == list(range(n))
    covered, stack, reached = [0] * n, [0], set()
    while stack:
        i = stack.pop()
        assert emitted(t, i)
        reached.add(i)
        for c in t.child[i]:
            if c < 0:
                covered[pos[~c]] += 1
            elif t.leaf[c]:
                f = first_position(t, c)
                assert t.count[c] <= LEAF_MAX
                below, s2 = [], [c]
                while s2:
                    for y in t.child[s2.pop()]:
                        if y >= 0:
                            s2.append(y)
                        else:
                            below.append(pos[~y])
                assert sorted(below) == list(range(f, f + t.count[c]))   # a leaf is a consecutive run
                for k in range(f, f + t.count[c]):
                    covered[k] += 1
            else:
                stack.append(c)
    assert reached == {i for i in range(n - 1) if emitted(t, i)}
    assert all(c == 1 for c in covered)
    return sah


@pytest.mark.parametrize("n", [2, 3, 9, 10, 17, 64, 300])
@pytest.mark.parametrize("duplicate_keys", [False, True])
def test_lbvh_index_logic(n, duplicate_keys):
    sah = build_and_check(n, seed=n, duplicate_keys=duplicate_keys)
    assert all(b <= a * 1.000001 for a, b in zip(sah, sah[1:]))
