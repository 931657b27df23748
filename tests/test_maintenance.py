"""Online tree maintenance, host logic (no GPU): the library's CompressionStatistics, GetEdges,
UpdateStatistics and OptimalTree against the oracle restatement, and the reference's own unit
scenarios (optimizer/optimal_tree_unittest.cpp, tree/compression_tree_unittest.cpp:296-342)."""
import numpy as np
import pytest

import oracle as OR
from oracle import maintenance as M

E = OR
I = OR.INT


@pytest.fixture(scope="module")
def G():
    import gputimeseriescompressionoptimizer_b200 as g
    g.lib()
    return g


def fake_tree():
    """optimal_tree_unittest.cpp:19-63: rle(dict(afl, delta(afl)), patch(scale(afl), patch(afl, afl))), Fix()ed"""
    n = M.Node
    root = n(E.RLE, I)
    left, right = n(E.DICT, I), n(E.PATCH, I)
    ll, lr = n(E.AFL, I), n(E.DELTA, I)
    lr.kids = [n(E.AFL, I)]
    left.kids = [ll, lr]
    rl, rr = n(E.SCALE, I), n(E.PATCH, I)
    rl.kids = [n(E.AFL, I)]
    rr.kids = [n(E.AFL, I), n(E.AFL, I)]
    right.kids = [rl, rr]
    root.kids = [left, right]
    return root.fix()


FAKE_STATS = [  # optimal_tree_unittest.cpp:65-135
    (0, E.RLE, E.DICT, 3), (0, E.RLE, E.PATCH, 2.5), (0, E.AFL, E.NONE, 2), (0, E.PATCH, E.DELTA, 1.5),
    (1, E.RLE, E.PATCH, 4), (1, E.RLE, E.DELTA, 1.5), (1, E.PATCH, E.SCALE, 1), (1, E.PATCH, E.PATCH, 2),
    (2, E.DICT, E.AFL, 3), (2, E.DELTA, E.AFL, 1), (3, E.DICT, E.DELTA, 2), (4, E.PATCH, E.SCALE, 2.5),
    (5, E.PATCH, E.PATCH, 3.5), (6, E.AFL, E.NONE, 4), (8, E.DELTA, E.AFL, 4.23), (10, E.SCALE, E.AFL, 3),
    (12, E.PATCH, E.AFL, 5), (13, E.PATCH, E.AFL, 1), (18, E.AFL, E.NONE, 4), (20, E.AFL, E.NONE, 8),
    (26, E.AFL, E.NONE, 11), (28, E.AFL, E.NONE, 12)]

CHANGES = {
    "edge_only": [(4, E.PATCH, E.DELTA, 1), (5, E.PATCH, E.DELTA, 4), (12, E.DELTA, E.AFL, 6)],
    "whole_node": [(2, E.PATCH, E.DELTA, 4), (3, E.PATCH, E.DICT, 4), (6, E.DELTA, E.AFL, 6),
                   (8, E.DICT, E.AFL, 5), (9, E.DICT, E.AFL, 5), (14, E.AFL, E.NONE, 6),
                   (16, E.AFL, E.NONE, 6), (17, E.AFL, E.NONE, 6)]}
EXPECT = {"edge_only": {12: (E.DELTA, E.AFL), 10: (E.SCALE, E.AFL)},
          "whole_node": {2: (E.PATCH, E.DELTA), 3: (E.PATCH, E.DICT)}}


def edge_types(nodes):
    nodes = np.asarray(nodes).reshape(-1, 2)
    return nodes


@pytest.mark.parametrize("case", ["edge_only", "whole_node"])
def test_optimal_tree_reference_scenarios(G, case):
    """OptimalTreeTest.Replace_FakedTree_FakedStats_right_{ReplaceEdgeOnly,WholeNode}"""
    root = fake_tree()
    root.ratio = 5.0
    nodes, ratios = M.nodes_of(root)
    # oracle
    st = M.Stats(5)
    for no, a, b, v in FAKE_STATS:
        st.set(no, (a, b), v)
    ot = M.OptimalTree(root, st)
    for no, a, b, v in CHANGES[case]:
        st.set(no, (a, b), v)
    root.ratio = 1.0
    assert ot.try_correct()
    got_o = {no: (a.enc, b.enc) for a, b, no in M.edges(ot.root)}
    # library
    gs = G.EdgeStats(5)
    for no, a, b, v in FAKE_STATS:
        gs.set(no, a, b, v)
    gt = G.OptimalTree(nodes, ratios, gs)
    for no, a, b, v in CHANGES[case]:
        gs.set(no, a, b, v)
    gt.set_ratio(0, 1.0)
    assert gt.try_correct()
    gnodes, gratios = gt.tree()
    pairs = np.asarray(gnodes).reshape(-1, 2)
    got_g = {no: (int(pairs[f][0]), int(pairs[t][0])) for no, f, t in G.tree_edges(gnodes)}
    for no, want in EXPECT[case].items():
        assert got_o[no] == want and got_g[no] == want
    onodes, oratios = M.nodes_of(ot.root)
    assert np.array_equal(gnodes, onodes) and np.array_equal(gratios, oratios)


def test_update_statistics_complex_tree(G):
    """CompressionTreeTest.UpdateStatistics_ComplexTree: scale(delta(patch(afl, afl))) compressed on
    an int column; edge 0 holds (scale, delta), edge 6 (patch, afl)."""
    rng = np.random.default_rng(7)
    x = (np.cumsum(rng.integers(-8, 9, 20000)) + 10 ** 6).astype(np.int32)
    root = M.tree_of(OR.tree_from_path([E.SCALE, E.DELTA, E.PATCH, E.AFL, E.NONE, E.AFL, E.NONE], I))
    M.compress_ratios(root, x)
    st = M.Stats(5)
    M.update_statistics(root, st)
    assert st.any(0)[0] == (E.SCALE, E.DELTA) and st.any(6)[0] == (E.PATCH, E.AFL)
    gs = G.EdgeStats(5)
    nodes, ratios = M.nodes_of(root)
    G.tree_update_statistics(nodes, ratios, gs)
    for no in range(62):
        assert gs.entries(no) == st.e[no]


def random_tree(rng, depth=0, dt=I):
    encs = [E.DELTA, E.SCALE, E.RLE, E.DICT, E.PATCH, E.CONST, E.AFL, E.GFC, E.NONE, E.FLOAT2INT, E.UNIQUE]
    enc = E.NONE if depth >= 4 or rng.random() < 0.25 else int(rng.choice(encs))
    n = M.Node(enc, dt, float(rng.choice([1.0, 1.5, 2.0, 3.25, 0.5])))
    n.kids = [random_tree(rng, depth + 1, M.return_type(enc, dt, j)) for j in range(M.N_RESULTS[enc])]
    return n


def random_stats(rng, st_o, st_g, k):
    encs = list(range(11))
    for _ in range(k):
        no = int(rng.integers(0, 62))
        a, b = int(rng.choice(encs)), int(rng.choice(encs))
        v = float(rng.choice([0.5, 1.0, 1.5, 2.0, 2.5, 3.0, 4.0]))  # repeated values exercise ties
        if rng.random() < 0.5:
            st_o.set(no, (a, b), v)
            st_g.set(no, a, b, v)
        else:
            st_o.update(no, (a, b), v)
            st_g.update(no, a, b, v)


def test_statistics_update_and_best(G):
    rng = np.random.default_rng(3)
    so, sg = M.Stats(5), G.EdgeStats(5)
    random_stats(rng, so, sg, 4000)
    for no in range(62):
        assert sg.entries(no) == so.e[no]
        for old in [(E.DELTA, E.AFL), (E.RLE, E.NONE), (E.PATCH, E.PATCH)]:
            for same in (False, True):
                assert sg.best(no, *old, same) == so.best(no, old, same)
    with pytest.raises(G.GtscError):
        sg.update(62, 0, 0, 1.0)


@pytest.mark.parametrize("seed", range(40))
def test_try_correct_random(G, seed):
    """Random trees and statistics: the same edges, correction decision, replacement and regrown
    subtree as the oracle restatement."""
    rng = np.random.default_rng(1000 + seed)
    dt = int(rng.choice([OR.INT, OR.FLOAT, OR.DOUBLE, OR.TIME]))
    root = random_tree(rng, dt=dt)
    if root.enc == E.NONE:
        root = M.Node(E.DELTA, dt, 2.0)
        root.kids = [random_tree(rng, 1, dt)]
    nodes, ratios = M.nodes_of(root)
    assert [(no, f, t) for no, f, t in G.tree_edges(nodes)] == \
        [(no, M.preorder(root).index(a), M.preorder(root).index(b)) for a, b, no in M.edges(root)]
    so, sg = M.Stats(5), G.EdgeStats(5)
    random_stats(rng, so, sg, 300)
    ot, gt = M.OptimalTree(root, so), G.OptimalTree(nodes, ratios, sg)
    for step in range(4):  # statistics drift, the root ratio falls, the tree is corrected
        random_stats(rng, so, sg, 60)
        r = float(rng.choice([0.9, 1.0, 1.2, 4.0]))
        ot.root.ratio = r
        gt.set_ratio(0, r)
        assert gt.try_correct() == ot.try_correct()
        gn, gr = gt.tree()
        on, orr = M.nodes_of(ot.root)
        assert np.array_equal(gn, on) and np.array_equal(gr, orr)
