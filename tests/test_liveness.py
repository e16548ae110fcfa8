"""Liveness maps, as the reference's test pins them
(sandbox/tests/test_liveness_computation.py:52-200)."""

from polymage_b200.liveness import compute_liveness


class Node(object):
    def __init__(self, name, parents=None):
        self.name = name
        self.parents = parents


def children_map(nodes):
    m = {}
    for n in nodes:
        for p in n.parents or []:
            m.setdefault(p, []).append(n)
    return m


def same(a, b):
    return set(a) == set(b) and all(set(a[k]) == set(b[k]) for k in a)


def test_chain():
    a = Node('a'); b = Node('b', [a]); c = Node('c', [b]); d = Node('d', [c])
    e = Node('e', [d]); f = Node('f', [e])
    nodes = [a, b, c, d, e, f]
    sched = dict((n, i) for i, n in enumerate(nodes))
    lm = compute_liveness(children_map(nodes), sched)
    assert same(lm, {1: [a], 2: [b], 3: [c], 4: [d], 5: [e]})


def test_chain_with_skips():
    a = Node('a'); b = Node('b', [a]); c = Node('c', [a, b])
    d = Node('d', [b, c]); e = Node('e', [c, d]); f = Node('f', [d, e])
    nodes = [a, b, c, d, e, f]
    sched = dict((n, i) for i, n in enumerate(nodes))
    lm = compute_liveness(children_map(nodes), sched)
    assert same(lm, {2: [a], 3: [b], 4: [c], 5: [d, e]})


def test_tree():
    a = Node('a'); b = Node('b', [a]); c = Node('c', [a])
    d = Node('d', [b]); e = Node('e', [b]); f = Node('f', [c])
    g = Node('g', [c])
    nodes = [a, b, c, d, e, f, g]
    sched = dict((n, i) for i, n in enumerate(nodes))
    lm = compute_liveness(children_map(nodes), sched)
    assert same(lm, {2: [a], 4: [b], 6: [c]})


def test_harris_two_schedules():
    img = Node('img'); Ix = Node('Ix', [img]); Iy = Node('Iy', [img])
    Ixx = Node('Ixx', [Ix]); Ixy = Node('Ixy', [Ix, Iy])
    Iyy = Node('Iyy', [Iy]); Sxx = Node('Sxx', [Ixx])
    Sxy = Node('Sxy', [Ixy]); Syy = Node('Syy', [Iyy])
    det = Node('det', [Sxx, Sxy, Syy]); trace = Node('trace', [Sxx, Syy])
    harris = Node('harris', [det, trace])
    nodes = [img, Ix, Iy, Ixx, Ixy, Iyy, Sxx, Sxy, Syy, det, trace, harris]
    cm = children_map(nodes)
    s1 = {img: 0, Ix: 1, Iy: 2, Ixx: 3, Ixy: 4, Iyy: 5, Sxx: 6, Sxy: 7,
          Syy: 8, det: 9, trace: 10, harris: 11}
    assert same(compute_liveness(cm, s1), {
        2: [img], 4: [Ix], 5: [Iy], 6: [Ixx], 7: [Ixy], 8: [Iyy],
        9: [Sxy], 10: [Sxx, Syy], 11: [det, trace]})
    s2 = {img: 0, Iy: 1, Iyy: 2, Syy: 3, Ix: 4, Ixy: 5, Sxy: 6, Ixx: 7,
          Sxx: 8, trace: 9, det: 10, harris: 11}
    assert same(compute_liveness(cm, s2), {
        3: [Iyy], 4: [img], 5: [Iy], 6: [Ixy], 7: [Ix], 8: [Ixx],
        10: [Sxx, Sxy, Syy], 11: [det, trace]})
