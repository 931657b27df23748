// optimizer.cpp -- online tree maintenance (host logic over the GPU tree compressor).
//
// Edge statistics: every compressed tree folds, for each of its edges, the mean of the two nodes'
// compression ratios into a running score per (edge number, parent encoding, child encoding):
// score = (max(score, 1) + max(ratio, 1)) / 2.  A full statistics update (the first part and every
// 10th after) folds in every FullStatisticsUpdate candidate of a 10 000-element sample and restarts
// from the best one; the parts in between are compressed with the current tree, whose own edges are
// folded in, and the tree is then corrected: when its ratio fell (or never exceeded 1), the first
// edge (breadth-first) whose score dropped or has a better alternative is replaced -- only the
// child when a better edge with the same parent exists, else the parent node -- and the replaced
// node's subtree is regrown from the best-scoring edges below it.
//
// Deviations from the reference, each where it has undefined behaviour or would write a blob it
// cannot decode: entries are scanned in (parent, child) order, so equal scores resolve to the
// smallest pair (the reference iterates an unordered_map); a node regrown below the last edge number
// gets `none` children instead of none at all (the reference would then emit a node with missing
// children, and reads statistics past their end at edge numbers 62 and 63); an encoding that cannot
// encode a node's data type (AFL of double) is never chosen.
#include "optimizer.hpp"

#include <queue>

namespace gtsc {

namespace {

bool encodable(int enc, int dt) { return !(enc == GTSC_AFL && dt == GTSC_DOUBLE); }

int flat_rec(FlatTree &f, const Tree &t, const std::vector<double> &r, int &i)
{
    if (i >= t.size()) fail(GTSC_ERR_ARG, "tree: incomplete node list");
    const int me = f.add(t.enc[i], t.dt[i], r.empty() ? 1.0 : r[i]);
    const int n = n_results(t.enc[i]);
    ++i;
    for (int j = 0; j < n; j++) {
        const int c = flat_rec(f, t, r, i);
        f.kids[me].push_back(c);
    }
    return me;
}

void pre_rec(const FlatTree &f, int k, Tree &t, std::vector<double> *r)
{
    t.enc.push_back(f.enc[k]);
    t.dt.push_back(f.dt[k]);
    if (r) r->push_back(f.ratio[k]);
    for (int c : f.kids[k]) pre_rec(f, c, t, r);
}

}  // namespace

// ------------------------------------------------------------------------------------ EdgeStats

EdgeStats::EdgeStats(int h) : height(h)
{
    if (h < 1 || h > 20) fail(GTSC_ERR_ARG, "edge statistics: tree height out of range");
    e.resize((size_t(1) << (h + 1)) - 2);
}

void EdgeStats::update(int no, EdgeType t, double ratio)
{
    if (no < 0 || no >= edges()) return;
    double &v = e[no][t];
    if (v < 1.0) v = 1.0;
    if (ratio < 1.0) ratio = 1.0;
    v += ratio;
    v /= 2.0;
}

void EdgeStats::set(int no, EdgeType t, double v)
{
    if (no < 0 || no >= edges()) fail(GTSC_ERR_ARG, "edge statistics: edge number out of range");
    e[no][t] = v;
}

double EdgeStats::get(int no, EdgeType t) const
{
    if (no < 0 || no >= edges()) return 0.0;
    auto it = e[no].find(t);
    return it == e[no].end() ? 0.0 : it->second;
}

EdgeStats::Best EdgeStats::best(int no, EdgeType old, bool same_beginning, int valid_dt, bool pick_parent) const
{
    Best b{EdgeType{old.first, GTSC_NONE}, 1.0};
    if (no < 0 || no >= edges()) return b;
    for (auto &kv : e[no]) {
        if (same_beginning && kv.first.first != old.first) continue;
        if (valid_dt >= 0 && !encodable(pick_parent ? kv.first.first : kv.first.second, valid_dt)) continue;
        if (kv.first.second != old.second && kv.second > b.value) b = Best{kv.first, kv.second};
    }
    return b;
}

EdgeStats::Best EdgeStats::any(int no) const
{
    Best b{EdgeType{0, 0}, 1.0};
    if (no < 0 || no >= edges()) return b;
    for (auto &kv : e[no]) b = Best{kv.first, kv.second};
    return b;
}

// ------------------------------------------------------------------------------------- FlatTree

int FlatTree::add(int e, int d, double r)
{
    enc.push_back((int16_t)e);
    dt.push_back((int16_t)d);
    ratio.push_back(r);
    kids.emplace_back();
    return (int)enc.size() - 1;
}

FlatTree FlatTree::from(const Tree &t, const std::vector<double> &ratios)
{
    FlatTree f;
    int i = 0;
    flat_rec(f, t, ratios, i);
    if (i != t.size()) fail(GTSC_ERR_ARG, "tree: extra nodes");
    return f;
}

Tree FlatTree::preorder(std::vector<double> *ratios) const
{
    Tree t;
    if (ratios) ratios->clear();
    if (!enc.empty()) pre_rec(*this, 0, t, ratios);
    return t;
}

std::vector<TreeEdge> tree_edges(const FlatTree &t, int height)
{
    std::vector<TreeEdge> out;
    if (t.enc.empty()) return out;
    const int max = (1 << (height + 1)) - 2;
    int no = 0;
    std::queue<int> q;  // -1: a missing child, numbered as if present
    q.push(0);
    while (!q.empty() && no < max) {
        const int el = q.front();
        q.pop();
        const int nk = el >= 0 ? (int)t.kids[el].size() : 0;
        for (int side = 0; side < 2; side++, no++) {
            if (nk > side) {
                out.push_back(TreeEdge{el, t.kids[el][side], no});
                q.push(t.kids[el][side]);
            } else {
                q.push(-1);
            }
        }
    }
    return out;
}

void update_statistics(const FlatTree &t, EdgeStats &st)
{
    for (auto &ed : tree_edges(t, st.height))
        st.update(ed.no, EdgeType{t.enc[ed.from], t.enc[ed.to]}, (t.ratio[ed.from] + t.ratio[ed.to]) / 2.0);
}

// ---------------------------------------------------------------------------------- OptimalTree

OptimalTree::OptimalTree(FlatTree t, std::shared_ptr<EdgeStats> stats)
    : tree(std::move(t)), live(std::move(stats))
{
    if (tree.enc.empty()) fail(GTSC_ERR_ARG, "optimal tree: empty tree");
    ratio = tree.ratio[0];
    snapshot = std::make_shared<EdgeStats>(*live);
    max_edge = (1 << (live->height + 1)) - 2;
}

void OptimalTree::replace(int node, const EdgeStats &st, int edge_no)
{
    const int e = tree.enc[node], d = tree.dt[node];
    const int r = n_results(e);
    if (edge_no > max_edge) {  // below the last edge number: `none` children (CompressionNode::Fix)
        for (int j = 0; j < r; j++) {
            const int c = tree.add(GTSC_NONE, d, 1.0);
            tree.kids[node].push_back(c);
        }
        return;
    }
    for (int i = 0; i < r; i++) {
        const int rt = return_type(e, d, i);
        const EdgeStats::Best b = st.best(edge_no + i, EdgeType{e, e}, false, rt, false);
        if (b.value > 1) {
            const int c = tree.add(b.type.second, rt, 1.0);
            tree.kids[node].push_back(c);
            replace(c, st, 2 * (edge_no + i) + 2);
        } else {
            const int c = tree.add(GTSC_NONE, rt, 1.0);
            tree.kids[node].push_back(c);
        }
    }
}

bool OptimalTree::try_correct()
{
    const double old_ratio = ratio, new_ratio = tree.ratio[0];
    if (old_ratio <= new_ratio && old_ratio > 1) return false;
    const EdgeStats &now = *live, &before = *snapshot;
    for (const TreeEdge &ed : tree_edges(tree, live->height)) {
        const EdgeType t{tree.enc[ed.from], tree.enc[ed.to]};
        const double ov = before.get(ed.no, t), nv = now.get(ed.no, t);
        const EdgeStats::Best best = now.best(ed.no, t, false, tree.dt[ed.from], true);
        if (!(nv < ov || best.value > nv)) continue;
        const EdgeStats::Best same = now.best(ed.no, t, true, tree.dt[ed.to], false);
        auto reset = [&](int k, int enc) {  // CompressionNode::Reset (tree/compression_node.cpp:225-241)
            tree.enc[k] = (int16_t)enc;
            tree.kids[k].clear();
            tree.ratio[k] = 1.0;
        };
        if (same.value > nv) {  // a better edge from the same parent: replace the child only
            reset(ed.to, same.type.second);
            replace(ed.to, now, 2 * (ed.no + 1));
        } else {                // replace the parent node
            reset(ed.from, best.type.first);
            replace(ed.from, now, ed.no % 2 ? ed.no - 1 : ed.no);
        }
        std::vector<double> r;
        const Tree pre = tree.preorder(&r);
        tree = FlatTree::from(pre, r);  // drop the detached nodes
        ratio = tree.ratio[0];
        snapshot = live;  // the reference keeps the live statistics from here on
        return true;
    }
    return false;
}

// ------------------------------------------------------------------------------------ Optimizer

DevBuf Optimizer::compress_data(View part, bool *full_update, bool *corrected, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    if (part.bytes % dtype_size(dt)) fail(GTSC_ERR_ARG, "optimizer: part is not a whole number of elements");
    const bool full = !opt || parts % 10 == 9;  // IsFullUpdateNeeded (:142-146)
    if (full) {
        const View sample(part.ptr, sample_bytes(dt, part.bytes));
        std::vector<Candidate> cands = plan_candidates(dt, sample, s);
        if (cands.empty()) fail(GTSC_ERR_ARG, "optimizer: no candidate tree");
        size_t bi = 0;
        for (size_t k = 0; k < cands.size(); k++) {
            update_statistics(FlatTree::from(cands[k].tree, cands[k].ratio), *stats);
            if (cands[k].ratio[0] > cands[bi].ratio[0]) bi = k;  // the first largest ratio
        }
        opt.reset(new OptimalTree(FlatTree::from(cands[bi].tree, cands[bi].ratio), stats));
    }
    const Tree t = opt->tree.preorder(nullptr);
    std::vector<double> r;
    DevBuf blob = tree_compress(t, part, s, &r);
    opt->tree = FlatTree::from(t, r);
    update_statistics(opt->tree, *stats);
    const bool corr = opt->try_correct();
    parts++;
    total_bytes += part.bytes;
    if (full_update) *full_update = full;
    if (corrected) *corrected = corr;
    return blob;
}

}  // namespace gtsc
