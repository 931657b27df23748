// planner.cpp -- the plain exhaustive planner over the GPU encodings.
//
// CompressionOptimizer::FullStatisticsUpdate (optimizer/compression_optimizer.cpp:88-140) enumerates
// every candidate tree reachable through PathGenerator::GetContinuations
// (optimizer/path_generator.cpp:93-146) by encoding the sample at each node and crossing the
// children's candidate lists; CompressData (:156-182) then Fix()es them and keeps the first one with
// the largest compression ratio.  Candidate sizes add up along the tree, so the first largest-ratio
// candidate is assembled from each child's first smallest candidate: this file evaluates exactly the
// same encodes and the same ordering without materialising the (up to 10^5) crossed trees.
#include "planner.hpp"

#include "tree.hpp"

namespace gtsc {

namespace {

constexpr int MAX_LEVEL = 3;  // optimizer/path_generator.cpp:15

// PathGenerator::GetContinuations (optimizer/path_generator.cpp:93-146).  `whole` = the input is a
// whole number of elements of its type; when it is not (a dictionary's code stream re-read as
// 8-byte values), every encoding but none would drop its last bytes (the reference's
// CastSharedCudaPtr), so only none is offered: a deliberate departure that keeps every planned
// tree lossless (the oracle does the same).
std::vector<int> continuations(int et, int dt, const Stats &st, int level, bool whole)
{
    std::vector<int> r;
    if (level != 0 && (et == GTSC_NONE || st.size == 0)) return r;
    r.push_back(GTSC_NONE);
    if (et == GTSC_AFL || et == GTSC_GFC || !whole) return r;
    if (level < MAX_LEVEL) {
        if (et != GTSC_DELTA) r.push_back(GTSC_DELTA);
        if (et != GTSC_SCALE && st.min != 0) r.push_back(GTSC_SCALE);
        if (et != GTSC_FLOAT_TO_INT && dt == GTSC_FLOAT) r.push_back(GTSC_FLOAT_TO_INT);
        if (et != GTSC_PATCH && et != GTSC_DICT) r.push_back(GTSC_PATCH);
        if (et != GTSC_DICT && et != GTSC_PATCH) r.push_back(GTSC_DICT);
        if (st.sorted || st.rl_metric >= 1.5f) {
            if (et != GTSC_CONST) r.push_back(GTSC_CONST);
            if (et != GTSC_RLE) r.push_back(GTSC_RLE);
        }
    }
    r.push_back(is_fp(dt) ? GTSC_GFC : GTSC_AFL);
    return r;
}

struct Cand {
    uint64_t size = UINT64_MAX;
    Tree tree;
};


void append(Tree &dst, const Tree &src)
{
    dst.enc.insert(dst.enc.end(), src.enc.begin(), src.enc.end());
    dst.dt.insert(dst.dt.end(), src.dt.begin(), src.dt.end());
}

// returns false when the reference would return an empty candidate list
bool fsu(View data, int et, int dt, int level, Cand &best, PlanCounters &ctr, cudaStream_t s)
{
    const Stats st = column_stats(dt, data, s);
    ctr.stats_calls++;
    const std::vector<int> cont = continuations(et, dt, st, level, data.bytes % dtype_size(dt) == 0);
    if (cont.empty()) return false;
    best.size = UINT64_MAX;
    for (int c : cont) {
        Parts p = encode(c, dt, data, s);
        ctr.encodes++;
        uint64_t psize = 8;
        for (auto &b : p) psize += b.bytes;
        const int r = n_results(c);
        Cand cand;
        bool ok = r > 0;
        Cand ch[2];
        for (int j = 0; j < r; j++)
            ok = fsu(View(p[j + 1]), c, return_type(c, dt, j), level + 1, ch[j], ctr, s) && ok;
        if (!ok) {
            cand.tree = leaf_tree(c, dt);
            cand.size = psize;
        } else {
            cand.tree.enc.push_back((int16_t)c);
            cand.tree.dt.push_back((int16_t)dt);
            cand.size = p[0].bytes + 8;
            for (int j = 0; j < r; j++) {
                append(cand.tree, ch[j].tree);
                cand.size += ch[j].size;
            }
        }
        if (cand.size < best.size) best = cand;
    }
    return true;
}

// FullStatisticsUpdate with every candidate kept (compression_optimizer.cpp:88-140, CrossTrees
// :38-78): per continuation, the crossed children candidates (left-major), or the bare node
void fsu_all(View data, int et, int dt, int level, std::vector<Candidate> &out, cudaStream_t s)
{
    const Stats st = column_stats(dt, data, s);
    for (int c : continuations(et, dt, st, level, data.bytes % dtype_size(dt) == 0)) {
        Parts p = encode(c, dt, data, s);
        uint64_t psize = 8;
        for (auto &b : p) psize += b.bytes;
        const int r = n_results(c);
        std::vector<Candidate> kid[2];
        bool crossed = r > 0;
        for (int j = 0; j < r; j++) {
            fsu_all(View(p[j + 1]), c, return_type(c, dt, j), level + 1, kid[j], s);
            crossed = crossed && !kid[j].empty();
        }
        auto make = [&](uint64_t size, const Candidate *a, const Candidate *b) {
            Candidate x;
            x.size = size;
            x.tree.enc.push_back((int16_t)c);
            x.tree.dt.push_back((int16_t)dt);
            x.ratio.push_back(compression_ratio(data.bytes, size));
            for (const Candidate *k : {a, b}) {
                if (!k) continue;
                append(x.tree, k->tree);
                x.ratio.insert(x.ratio.end(), k->ratio.begin(), k->ratio.end());
            }
            out.push_back(std::move(x));
        };
        if (!crossed) {  // CompressNode::Fix gives the bare node `none` children of its own type
            Candidate x;
            x.size = psize;
            x.tree = leaf_tree(c, dt);
            x.ratio.assign(x.tree.size(), 1.0);
            x.ratio[0] = compression_ratio(data.bytes, psize);
            out.push_back(std::move(x));
        } else if (r == 1) {
            for (auto &a : kid[0]) make(a.size + p[0].bytes + 8, &a, nullptr);
        } else {
            for (auto &a : kid[0])
                for (auto &b : kid[1]) make(a.size + b.size + p[0].bytes + 8, &a, &b);
        }
    }
}

// PathGenerator::GeneratePaths (optimizer/path_generator.cpp:20-68): 6 x 5 paths
std::vector<std::vector<int16_t>> generate_paths()
{
    const std::vector<std::vector<int16_t>> first = {
        {}, {GTSC_FLOAT_TO_INT}, {GTSC_DELTA}, {GTSC_SCALE}, {GTSC_DELTA, GTSC_FLOAT_TO_INT},
        {GTSC_SCALE, GTSC_FLOAT_TO_INT}};
    const std::vector<std::vector<int16_t>> second = {
        {GTSC_DICT, GTSC_AFL, GTSC_NONE, GTSC_AFL, GTSC_NONE},
        {GTSC_CONST, GTSC_AFL, GTSC_NONE},
        {GTSC_RLE, GTSC_AFL, GTSC_NONE, GTSC_AFL, GTSC_NONE},
        {GTSC_AFL, GTSC_NONE},
        {GTSC_PATCH, GTSC_AFL, GTSC_NONE, GTSC_AFL, GTSC_NONE}};
    std::vector<std::vector<int16_t>> out;
    for (auto &a : first)
        for (auto &b : second) {
            std::vector<int16_t> p = a;
            p.insert(p.end(), b.begin(), b.end());
            out.push_back(p);
        }
    return out;
}

}  // namespace

uint64_t sample_bytes(int dt, uint64_t bytes)
{
    const uint64_t es = dtype_size(dt);
    if (!es) return 0;
    const uint64_t n = bytes / es;
    return n <= 10000 ? bytes : 10000 * es;  // compression_optimizer.cpp:148-154
}

Tree plan_exhaustive(int dt, View sample, uint64_t *best_size, PlanCounters *counters, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    PlanCounters ctr;
    Cand best;
    fsu(sample, GTSC_NONE, dt, 0, best, ctr, s);
    // max_element over GetCompressionRatio: ratios saturate at 1.0, so only a candidate strictly
    // smaller than the sample beats the leading `none` tree
    if (!(best.size < sample.bytes)) {
        best.tree = leaf_tree(GTSC_NONE, dt);
        best.size = sample.bytes + 16;
    }
    if (best_size) *best_size = best.size;
    if (counters) *counters = ctr;
    return best.tree;
}

std::vector<Candidate> plan_candidates(int dt, View sample, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    std::vector<Candidate> out;
    fsu_all(sample, GTSC_NONE, dt, 0, out, s);
    return out;
}

Tree optimize_tree(int dt, View data, uint64_t *best_size, cudaStream_t s)
{
    if (!dtype_size(dt)) fail(GTSC_ERR_ARG, "unknown data type");
    uint64_t min_size = data.bytes;
    Tree result = leaf_tree(GTSC_NONE, dt);
    for (auto &path : generate_paths()) {
        Tree t = tree_from_path(path.data(), (int)path.size(), dt);
        uint64_t sz;
        try {
            sz = tree_predict_size(t, data, s);
        } catch (const Error &e) {
            if (e.code == GTSC_ERR_UNSUPPORTED || e.code == GTSC_ERR_TYPE) continue;  // reference throws
            throw;
        }
        if (sz < min_size) {
            min_size = sz;
            result = t;
        }
    }
    if (best_size) *best_size = min_size;
    return result;
}

}  // namespace gtsc
