"""CPU check of the counting identity behind the tree program's same-label
blocks (csrc/treecount.cu): for a tree query whose same-label vertices are
siblings or grandparent and grandchild,

    embeddings = sum over partitions pi of each label's vertices into blocks of
                 pairwise non-adjacent vertices of  mu(pi) * hom(Q / pi),
    mu(pi)     = prod over blocks of (-1)^(|B|-1) (|B|-1)!

where an embedding is a label-preserving map onto data edges that is
injective on same-label non-adjacent pairs (the pairs the enumeration checks),
and hom(Q / pi) counts label-preserving edge-preserving maps of the quotient
(one data vertex per block; parallel edges are one constraint).  Embeddings
are counted by brute force, hom(Q / pi) by a bottom-up program over the
quotient tree, on small seeded random graphs."""
import itertools
import math
import random

import pytest


def random_graph(n, p, nlabels, seed):
    rng = random.Random(seed)
    labels = [rng.randrange(nlabels) for _ in range(n)]
    adj = [set() for _ in range(n)]
    for a in range(n):
        for b in range(a + 1, n):
            if rng.random() < p:
                adj[a].add(b)
                adj[b].add(a)
    return labels, adj


def brute_embeddings(qlab, qedges, glab, gadj):
    n = len(qlab)
    qadj = [set() for _ in range(n)]
    for a, b in qedges:
        qadj[a].add(b)
        qadj[b].add(a)
    cands = [[v for v in range(len(glab)) if glab[v] == qlab[u]] for u in range(n)]
    total = 0
    for m in itertools.product(*cands):
        if any(m[b] not in gadj[m[a]] for a, b in qedges):
            continue
        if any(m[a] == m[b] for a in range(n) for b in range(a + 1, n)
               if qlab[a] == qlab[b] and b not in qadj[a]):
            continue
        total += 1
    return total


def partitions(qlab, qadj):
    """Set partitions of each label's vertices into blocks of pairwise
    non-adjacent vertices, as a block id per vertex."""
    n = len(qlab)
    out = []

    def place(u, block, members):
        if u == n:
            out.append(list(block))
            return
        for b, m in enumerate(members):
            if qlab[m[0]] == qlab[u] and not any(w in qadj[u] for w in m):
                m.append(u)
                block[u] = b
                place(u + 1, block, members)
                m.pop()
        block[u] = len(members)
        members.append([u])
        place(u + 1, block, members)
        members.pop()

    place(0, [0] * n, [])
    return out


def mu(block):
    sizes = {}
    for b in block:
        sizes[b] = sizes.get(b, 0) + 1
    c = 1
    for s in sizes.values():
        c *= (-1) ** (s - 1) * math.factorial(s - 1)
    return c


def hom_quotient_tree(qlab, qedges, block, glab, gadj):
    """Homomorphisms of the quotient by `block` (None if it is not a tree):
    w_B(v) = prod over child blocks C of sum over neighbours v' of v with
    label l(C) of w_C(v'), counted from the block of vertex 0."""
    nb = max(block) + 1
    lab = [None] * nb
    for u, b in enumerate(block):
        lab[b] = qlab[u]
    qe = {(min(block[a], block[b]), max(block[a], block[b])) for a, b in qedges}
    if any(a == b for a, b in qe) or len(qe) != nb - 1:
        return None
    badj = [set() for _ in range(nb)]
    for a, b in qe:
        badj[a].add(b)
        badj[b].add(a)

    def weight(B, parent, v):
        w = 1
        for C in badj[B]:
            if C == parent:
                continue
            w *= sum(weight(C, B, x) for x in gadj[v] if glab[x] == lab[C])
        return w

    root = block[0]
    return sum(weight(root, None, v) for v in range(len(glab)) if glab[v] == lab[root])


TREES = [
    # (labels, edges): stars and paths with same-label siblings or
    # grandparent/grandchild pairs, including blocks of three
    ([0, 1, 1, 1], [(0, 1), (0, 2), (0, 3)]),
    ([0, 1, 0, 2], [(0, 1), (1, 2), (2, 3)]),
    ([0, 1, 0, 1], [(0, 1), (1, 2), (2, 3)]),
    ([0, 1, 1, 0, 0, 2], [(0, 1), (0, 2), (1, 3), (1, 4), (0, 5)]),
    ([1, 0, 1, 1, 0], [(0, 1), (1, 2), (1, 3), (3, 4)]),
]


@pytest.mark.parametrize("seed", [3, 17])
@pytest.mark.parametrize("qlab,qedges", TREES)
def test_block_inclusion_exclusion_matches_brute_force(qlab, qedges, seed):
    glab, gadj = random_graph(16, 0.6, 3, seed)
    n = len(qlab)
    qadj = [set() for _ in range(n)]
    for a, b in qedges:
        qadj[a].add(b)
        qadj[b].add(a)
    parts = partitions(qlab, qadj)
    total = 0
    for block in parts:
        h = hom_quotient_tree(qlab, qedges, block, glab, gadj)
        assert h is not None  # every quotient of these shapes is a tree
        total += mu(block) * h
    assert total == brute_embeddings(qlab, qedges, glab, gadj)
    # the graph has matches, and the same-label blocks take some away
    assert 0 < total < hom_quotient_tree(qlab, qedges, list(range(n)), glab, gadj)


def test_far_same_label_pair_gives_a_cyclic_quotient():
    """Same-label vertices three edges apart merge into a triangle: the tree
    program leaves such queries to the enumeration."""
    qlab, qedges = [0, 1, 2, 0], [(0, 1), (1, 2), (2, 3)]
    qadj = [set() for _ in range(4)]
    for a, b in qedges:
        qadj[a].add(b)
        qadj[b].add(a)
    glab, gadj = random_graph(8, 0.5, 3, 5)
    cyclic = [b for b in partitions(qlab, qadj)
              if hom_quotient_tree(qlab, qedges, b, glab, gadj) is None]
    assert cyclic == [[0, 1, 2, 0]]
