"""Subtree-checkpoint plans (h3g_checkpoint_plan, host only).

The plan cuts a tree into blocks rooted at checkpoint nodes; checkpoint nodes own persistent
partial slots, every other node a scratch slot shared with the nodes of other blocks.  These tests
check the plan's invariants and replay the evaluation order the engine runs over it (inside pass
by blocks in post-order; outside pass by blocks in reverse post-order, each recomputing its inside
partials below its root, walking its nodes by depth and accumulating its branches), asserting that
every read of a slot finds the partial of the node it wants.  The device kernels read and write
exactly these slots (Topo::iidx / Topo::vidx), so a plan that passes here cannot alias two live
partials on the GPU.
"""
import numpy as np
import pytest

from hyphy3 import _capi


def _random_tree(rng, n_leaves, max_children=2):
    """Random rooted tree: parent array and leaf flags (node 0 is the root)."""
    parent = [-1]
    open_nodes = [0]
    n_kids = {0: 0}
    # grow by attaching children to random open nodes until enough childless nodes exist
    while sum(1 for i in range(len(parent)) if n_kids.get(i, 0) == 0) < n_leaves:
        u = open_nodes[rng.integers(len(open_nodes))]
        parent.append(u)
        v = len(parent) - 1
        n_kids[u] = n_kids.get(u, 0) + 1
        n_kids[v] = 0
        if n_kids[u] >= max_children:
            open_nodes.remove(u)
        open_nodes.append(v)
    n = len(parent)
    kids = [[] for _ in range(n)]
    for v in range(1, n):
        kids[parent[v]].append(v)
    is_leaf = np.array([len(kids[v]) == 0 for v in range(n)], dtype=np.uint8)
    return np.array(parent, dtype=np.int32), is_leaf


def _yule(rng, n_leaves):
    return _random_tree(rng, n_leaves, 2)


def _caterpillar(n_leaves):
    parent, leaf = [-1], [0]
    spine = 0
    for k in range(n_leaves - 1):
        parent.append(spine)
        leaf.append(1)
        if k < n_leaves - 2:
            parent.append(spine)
            leaf.append(0)
            spine = len(parent) - 1
        else:
            parent.append(spine)
            leaf.append(1)
    return np.array(parent, dtype=np.int32), np.array(leaf, dtype=np.uint8)


def _structure(parent, is_leaf):
    n = len(parent)
    kids = [[] for _ in range(n)]
    root = int(np.flatnonzero(parent < 0)[0])
    for v in range(n):
        if parent[v] >= 0:
            kids[parent[v]].append(v)
    depth = np.full(n, -1)
    depth[root] = 0
    order = [root]
    for u in order:
        for c in kids[u]:
            depth[c] = depth[u] + 1
            order.append(c)
    height = np.zeros(n, dtype=int)
    for u in reversed(order):
        for c in kids[u]:
            height[u] = max(height[u], height[c] + 1)
    return root, kids, depth, height


def _replay(parent, is_leaf, plan):
    """Run the engine's evaluation order over the plan's slots; assert every read is the wanted node's."""
    root, kids, depth, height = _structure(parent, is_leaf)
    n = len(parent)
    ck, blk = plan["is_checkpoint"], plan["block"]
    si, sv = plan["slot_internal"], plan["slot_vf"]
    nb = plan["blocks"]
    D, Ms, U, Vf = {}, {}, {}, {}              # slot -> node whose partial it holds
    members = [[] for _ in range(nb)]
    for v in range(n):
        members[blk[v]].append(v)
    broot = [None] * nb
    for v in range(n):
        if ck[v]:
            broot[blk[v]] = v
    inner = lambda b: sorted((v for v in members[b] if not is_leaf[v]), key=lambda v: height[v])

    def inside(b, with_root):
        for u in inner(b):
            if u == broot[b] and not with_root:
                continue
            for c in kids[u]:
                if not is_leaf[c]:
                    assert Ms[si[c]] == c, f"inside of {u} reads the message of {Ms[si[c]]} for child {c}"
            D[si[u]] = u
            Ms[si[u]] = u

    for b in range(nb):
        inside(b, True)
    assert D[si[root]] == root                  # the root read
    accumulated = set()
    for b in reversed(range(nb)):
        if b != nb - 1:
            inside(b, False)
        for u in sorted((v for v in members[b] if not is_leaf[v]), key=lambda v: depth[v]):
            if u != root:
                assert U[si[u]] == u, f"outside of the children of {u} reads U of {U[si[u]]}"
            assert D[si[u]] == u                  # its own exponents (Eown) live beside D
            for c in kids[u]:
                for s in kids[u]:
                    if s != c and not is_leaf[s]:
                        assert Ms[si[s]] == s, f"child {c} of {u} reads the message of {Ms[si[s]]} for sibling {s}"
                # the mixed path scales the gradient operand by the exponents of D_root and D_c
                assert D[si[root]] == root
                if not is_leaf[c]:
                    assert D[si[c]] == c, f"child {c} of {u} reads the inside partial of {D[si[c]]}"
                Vf[sv[c]] = c
                if not is_leaf[c]:
                    U[si[c]] = c
        for v in members[b]:
            if v == root:
                continue
            assert Vf[sv[v]] == v, f"branch {v} reads the gradient operand of {Vf[sv[v]]}"
            if not is_leaf[v]:
                assert D[si[v]] == v, f"branch {v} reads the inside partial of {D[si[v]]}"
            accumulated.add(v)
    assert accumulated == set(range(n)) - {root}


def _check_invariants(parent, is_leaf, target, plan):
    root, kids, depth, height = _structure(parent, is_leaf)
    n = len(parent)
    ck, blk = plan["is_checkpoint"], plan["block"]
    ncp = plan["persistent"]
    assert ck[root] == 1
    assert plan["blocks"] == ncp == int(ck.sum())
    assert blk[root] == plan["blocks"] - 1                        # the root's block last
    for v in range(n):
        if ck[v]:
            assert 0 <= plan["slot_internal"][v] < ncp and plan["slot_vf"][v] == plan["slot_internal"][v]
            if v != root:
                assert blk[parent[v]] > blk[v]                     # blocks in post-order
        else:
            assert blk[v] == blk[parent[v]]
            assert plan["slot_vf"][v] >= ncp
            if is_leaf[v]:
                assert plan["slot_internal"][v] == -1
            else:
                assert ncp <= plan["slot_internal"][v] < ncp + plan["scratch_internal"]
            assert plan["slot_vf"][v] < ncp + plan["scratch_nodes"]
    max_kids = max(len(k) for k in kids)
    for b in range(plan["blocks"]):
        size = int((blk == b).sum())
        assert size <= 1 + max_kids * (max(target, 2) - 1)
        nodes = np.flatnonzero(blk == b)
        for key in ("slot_internal", "slot_vf"):
            sl = [plan[key][v] for v in nodes if plan[key][v] >= ncp]
            assert len(sl) == len(set(sl))
    assert ncp + plan["scratch_internal"] <= int((is_leaf == 0).sum())
    assert ncp + plan["scratch_nodes"] <= n


@pytest.mark.parametrize("target", [2, 3, 8, 40, 1000000])
def test_plan_on_random_trees(target):
    rng = np.random.default_rng(7 + target % 97)
    for maker in (lambda: _yule(rng, 60), lambda: _random_tree(rng, 50, 4), lambda: _caterpillar(40),
                  lambda: _yule(rng, 300)):
        parent, is_leaf = maker()
        plan = _capi.checkpoint_plan(parent, is_leaf, target)
        _check_invariants(parent, is_leaf, target, plan)
        _replay(parent, is_leaf, plan)


def test_single_block_when_target_exceeds_tree():
    rng = np.random.default_rng(3)
    parent, is_leaf = _yule(rng, 100)
    plan = _capi.checkpoint_plan(parent, is_leaf, len(parent) + 1)
    assert plan["blocks"] == 1
    assert plan["persistent"] + plan["scratch_internal"] == int((is_leaf == 0).sum())
    assert plan["persistent"] + plan["scratch_nodes"] == len(parent)


def test_plan_shrinks_the_slot_count_on_a_1024_taxon_tree():
    rng = np.random.default_rng(11)
    parent, is_leaf = _yule(rng, 1024)
    full = int((is_leaf == 0).sum()) * 3 + len(parent)             # D, Ms, U per internal node + one Vf per node
    best = min(3 * (p["persistent"] + p["scratch_internal"]) + p["persistent"] + p["scratch_nodes"]
               for p in (_capi.checkpoint_plan(parent, is_leaf, t) for t in (16, 32, 64, 128)))
    assert best * 5 < full                                          # at least 5x fewer partial vectors
    _replay(parent, is_leaf, _capi.checkpoint_plan(parent, is_leaf, 64))


def test_plan_rejects_bad_trees():
    with pytest.raises(_capi.H3GError):
        _capi.checkpoint_plan(np.array([-1, -1, 0], dtype=np.int32), np.array([0, 0, 1], dtype=np.uint8), 4)
    with pytest.raises(_capi.H3GError):
        _capi.checkpoint_plan(np.array([-1, 0, 1], dtype=np.int32), np.array([0, 1, 1], dtype=np.uint8), 4)
