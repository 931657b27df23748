"""Online tree maintenance restated in Python over the oracle's encoders.

TEST INFRASTRUCTURE ONLY (imported by tests/): the checker of the library's CompressionStatistics /
OptimalTree / CompressData implementation, never part of the product.

Restates:
  CompressionStatistics::Update / Get / GetBest / GetAny   tree/compression_statistics.cpp:31-104
  CompressionTree::GetEdges / UpdateStatistics             tree/compression_tree.cpp:199-240
  CompressionNode::Compress (node ratios), Fix, Reset      tree/compression_node.cpp:103-135, 209-241
  OptimalTree::Replace / TryCorrectTree                    optimizer/optimal_tree.cpp:14-93
  CompressionOptimizer::FullStatisticsUpdate / CrossTrees  optimizer/compression_optimizer.cpp:38-140
  CompressionOptimizer::CompressData                       optimizer/compression_optimizer.cpp:142-193
  PathGenerator::GetContinuations                          optimizer/path_generator.cpp:93-146
    (an input that is not a whole number of elements is offered only none)

Fixed choices where the reference is unordered or undefined (the same ones the library makes):
statistics entries are scanned in (parent, child) order; a node regrown below the last edge number
gets `none` children; AFL is never chosen for a double node.
"""
import copy
from collections import deque

import numpy as np

import oracle as OR

N_RESULTS = {OR.DELTA: 1, OR.AFL: 1, OR.SCALE: 1, OR.UNIQUE: 1, OR.FLOAT2INT: 1, OR.CONST: 1,
             OR.RLE: 2, OR.DICT: 2, OR.PATCH: 2, OR.GFC: 2, OR.NONE: 0}


def return_type(enc, dt, j):
    """Encoding::GetReturnTypes (rle {int, T}, floatToInt {int}, others {T, T})."""
    if enc == OR.RLE and j == 0:
        return OR.INT
    if enc == OR.FLOAT2INT:
        return OR.INT
    return dt


def ratio(inp, out):
    """Encoding::GetCompressionRatio (compression/encoding.hpp:78-84)."""
    return 1.0 if out <= 0 or out > inp else inp / out


def encodable(enc, dt):
    return not (enc == OR.AFL and dt == OR.DOUBLE)


class Node:
    def __init__(self, enc, dt, r=1.0):
        self.enc, self.dt, self.ratio, self.kids = enc, dt, r, []

    def fix(self):
        """CompressionNode::Fix: leaves get `none` children of the node's own type."""
        if not self.kids:
            self.kids = [Node(OR.NONE, self.dt) for _ in range(N_RESULTS[self.enc])]
        else:
            for k in self.kids:
                k.fix()
        return self


def preorder(root):
    out = []

    def rec(n):
        out.append(n)
        for k in n.kids:
            rec(k)
    rec(root)
    return out


def nodes_of(root):
    """pre-order (encoding, dtype) pairs as the library's int16 node list, and the ratios"""
    pre = preorder(root)
    return (np.array([v for n in pre for v in (n.enc, n.dt)], np.int16),
            np.array([n.ratio for n in pre], np.float64))


def tree_of(nodes, ratios=None):
    nodes = np.asarray(nodes).reshape(-1, 2)
    pos = [0]

    def rec():
        k = pos[0]
        pos[0] += 1
        n = Node(int(nodes[k][0]), int(nodes[k][1]), 1.0 if ratios is None else float(ratios[k]))
        n.kids = [rec() for _ in range(N_RESULTS[n.enc])]
        return n
    return rec()


class Stats:
    """CompressionStatistics(height): 2^(h+1) - 2 edges of {(parent, child): score}"""

    def __init__(self, height=5):
        self.height = height
        self.e = [dict() for _ in range((1 << (height + 1)) - 2)]

    def update(self, no, t, r):
        if not 0 <= no < len(self.e):
            return
        v = self.e[no].get(t, 0.0)
        if v < 1.0:
            v = 1.0
        if r < 1.0:
            r = 1.0
        self.e[no][t] = (v + r) / 2.0

    def set(self, no, t, v):
        self.e[no][t] = v

    def get(self, no, t):
        return self.e[no].get(t, 0.0) if 0 <= no < len(self.e) else 0.0

    def best(self, no, old, same=False, valid_dt=-1, pick_parent=False):
        b = ((old[0], OR.NONE), 1.0)
        if not 0 <= no < len(self.e):
            return b
        for t in sorted(self.e[no]):
            if same and t[0] != old[0]:
                continue
            if valid_dt >= 0 and not encodable(t[0] if pick_parent else t[1], valid_dt):
                continue
            if t[1] != old[1] and self.e[no][t] > b[1]:
                b = (t, self.e[no][t])
        return b

    def any(self, no):
        b = ((0, 0), 1.0)
        for t in sorted(self.e[no]):
            b = (t, self.e[no][t])
        return b


def edges(root, height=5):
    """CompressionTree::GetEdges: breadth-first, missing children numbered as if present"""
    out, no, mx = [], 0, (1 << (height + 1)) - 2
    q = deque([root])
    while q and no < mx:
        el = q.popleft()
        kids = el.kids if el is not None else []
        for side in range(2):
            if len(kids) > side:
                out.append((el, kids[side], no))
                q.append(kids[side])
            else:
                q.append(None)
            no += 1
    return out


def update_statistics(root, st):
    for a, b, no in edges(root, st.height):
        st.update(no, (a.enc, b.enc), (a.ratio + b.ratio) / 2.0)


class OptimalTree:
    def __init__(self, root, live):
        self.root, self.ratio, self.live = root, root.ratio, live
        self.snapshot = copy.deepcopy(live)
        self.max_edge = (1 << (live.height + 1)) - 2

    def replace(self, node, st, edge_no):
        r = N_RESULTS[node.enc]
        if edge_no > self.max_edge:
            node.kids = [Node(OR.NONE, node.dt) for _ in range(r)]
            return
        for i in range(r):
            rt = return_type(node.enc, node.dt, i)
            t, v = st.best(edge_no + i, (node.enc, node.enc), False, rt, False)
            if v > 1:
                c = Node(t[1], rt)
                node.kids.append(c)
                self.replace(c, st, 2 * (edge_no + i) + 2)
            else:
                node.kids.append(Node(OR.NONE, rt))

    def try_correct(self):
        old, new = self.ratio, self.root.ratio
        if old <= new and old > 1:
            return False
        for a, b, no in edges(self.root, self.live.height):
            t = (a.enc, b.enc)
            ov, nv = self.snapshot.get(no, t), self.live.get(no, t)
            best = self.live.best(no, t, False, a.dt, True)
            if not (nv < ov or best[1] > nv):
                continue
            same = self.live.best(no, t, True, b.dt, False)
            if same[1] > nv:
                b.enc, b.kids, b.ratio = same[0][1], [], 1.0
                self.replace(b, self.live, 2 * (no + 1))
            else:
                a.enc, a.kids, a.ratio = best[0][0], [], 1.0
                self.replace(a, self.live, no - 1 if no % 2 else no)
            self.ratio = self.root.ratio
            self.snapshot = self.live
            return True
        return False


def continuations(et, dt, st, level, max_level=3, whole=True):
    """`whole`: the input is a whole number of elements of its type; when it is not (a dictionary's
    code stream re-read as 8-byte values) only none is offered, as the library's planner does."""
    r = []
    if level != 0 and (et == OR.NONE or st.size == 0):
        return r
    r.append(OR.NONE)
    if et in (OR.AFL, OR.GFC) or not whole:
        return r
    if level < max_level:
        if et != OR.DELTA:
            r.append(OR.DELTA)
        if et != OR.SCALE and st.min != 0:
            r.append(OR.SCALE)
        if et != OR.FLOAT2INT and dt == OR.FLOAT:
            r.append(OR.FLOAT2INT)
        if et not in (OR.PATCH, OR.DICT):
            r.append(OR.PATCH)
        if et not in (OR.DICT, OR.PATCH):
            r.append(OR.DICT)
        if st.sorted or st.rl_metric >= 1.5:
            if et != OR.CONST:
                r.append(OR.CONST)
            if et != OR.RLE:
                r.append(OR.RLE)
    r.append(OR.GFC if dt in (OR.FLOAT, OR.DOUBLE) else OR.AFL)
    return r


def candidates(data, dt, et=OR.NONE, level=0):
    """FullStatisticsUpdate: [(root Node, size)] with every node's ratio, un-Fixed"""
    data = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    st = OR.stats(dt, data)
    out = []
    for c in continuations(et, dt, st, level, whole=data.size % OR.NP_TYPES[dt]().itemsize == 0):
        parts = OR.encode(c, dt, data)
        psize = 8 + sum(p.size for p in parts)
        r = N_RESULTS[c]
        kids = [candidates(parts[j + 1], return_type(c, dt, j), c, level + 1) for j in range(r)]
        part = []
        if r == 1 and kids[0]:
            for k, ks in kids[0]:
                size = ks + parts[0].size + 8
                n = Node(c, dt, ratio(data.size, size))
                n.kids = [copy.deepcopy(k)]
                part.append((n, size))
        elif r == 2 and kids[0] and kids[1]:
            for k0, s0 in kids[0]:
                for k1, s1 in kids[1]:
                    size = s0 + s1 + parts[0].size + 8
                    n = Node(c, dt, ratio(data.size, size))
                    n.kids = [copy.deepcopy(k0), copy.deepcopy(k1)]
                    part.append((n, size))
        if not part:
            part = [(Node(c, dt, ratio(data.size, psize)), psize)]
        out.extend(part)
    return out


def compress_ratios(root, data):
    """CompressionNode::Compress: sets each node's ratio; returns the subtree's output bytes"""
    data = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    if root.enc == OR.NONE:
        out = 16 + data.size
    else:
        parts = OR.encode(root.enc, root.dt, data)
        out = 8 + parts[0].size + sum(compress_ratios(k, parts[j + 1]) for j, k in enumerate(root.kids))
    root.ratio = ratio(data.size, out)
    return out


class Optimizer:
    """CompressionOptimizer::CompressData for one column"""

    def __init__(self, dt):
        self.dt, self.stats, self.opt, self.parts = dt, Stats(5), None, 0

    def compress(self, x):
        x = np.ascontiguousarray(x)
        full = self.opt is None or self.parts % 10 == 9
        if full:
            es = x.itemsize
            sample = x[:OR.sample_bytes(self.dt, x.nbytes) // es]
            cands = [n.fix() for n, _ in candidates(sample, self.dt)]
            best = None
            for n in cands:
                update_statistics(n, self.stats)
                if best is None or n.ratio > best.ratio:
                    best = n
            self.opt = OptimalTree(best, self.stats)
        nodes, _ = nodes_of(self.opt.root)
        blob = OR.tree_compress(nodes, x)
        compress_ratios(self.opt.root, x)
        update_statistics(self.opt.root, self.stats)
        corrected = self.opt.try_correct()
        self.parts += 1
        return blob, full, corrected
