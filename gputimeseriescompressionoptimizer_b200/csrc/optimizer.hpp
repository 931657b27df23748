// optimizer.hpp -- online tree maintenance: the edge statistics of compression trees
// (CompressionStatistics, tree/compression_statistics.cpp), the tree correction of OptimalTree
// (optimizer/optimal_tree.cpp) and the chunk loop of CompressionOptimizer::CompressData
// (optimizer/compression_optimizer.cpp:142-193).
#pragma once

#include "common.cuh"
#include "planner.hpp"
#include "tree.hpp"

#include <map>
#include <memory>

namespace gtsc {

using EdgeType = std::pair<int, int>;  // (encoding of the parent, encoding of the child)

// CompressionStatistics: per edge number (breadth-first over a full binary tree of the given height,
// 2^(h+1) - 2 edges) a running score of each edge type.  Entries are kept in (parent, child)
// order, which fixes the tie order of best() (the reference iterates a hash map).
struct EdgeStats {
    int height = 5;
    std::vector<std::map<EdgeType, double>> e;
    explicit EdgeStats(int h = 5);
    int edges() const { return (int)e.size(); }
    void update(int no, EdgeType t, double ratio);    // Update (:31-46)
    void set(int no, EdgeType t, double v);           // Set (:151-154)
    double get(int no, EdgeType t) const;             // Get (:101-104); 0 when absent
    struct Best {
        EdgeType type;
        double value;
    };
    // GetBest (:61-81): the first entry with the highest score above 1 whose child differs from
    // old.second (and, with same_beginning, whose parent is old.first); (old.first, none, 1) if none.
    // valid_dt >= 0 also skips entries whose chosen encoding (the parent when pick_parent, else the
    // child) cannot encode that data type.
    Best best(int no, EdgeType old, bool same_beginning, int valid_dt = -1, bool pick_parent = false) const;
    Best any(int no) const;                           // GetAny (:48-59): the last entry
};

// a tree whose nodes can be replaced in place: node k has children kids[k]; root = node 0
struct FlatTree {
    std::vector<int16_t> enc, dt;
    std::vector<double> ratio;
    std::vector<std::vector<int>> kids;
    int add(int e, int d, double r);
    static FlatTree from(const Tree &t, const std::vector<double> &ratios);
    Tree preorder(std::vector<double> *ratios) const;
};

struct TreeEdge {
    int from, to, no;
};
// CompressionTree::GetEdges (tree/compression_tree.cpp:199-230)
std::vector<TreeEdge> tree_edges(const FlatTree &t, int height = 5);
// CompressionTree::UpdateStatistics (:232-240): edge score = mean of the two nodes' ratios
void update_statistics(const FlatTree &t, EdgeStats &st);

// OptimalTree (optimizer/optimal_tree.hpp:24-63, optimal_tree.cpp)
struct OptimalTree {
    FlatTree tree;
    double ratio = 1.0;                  // the tree's ratio when last built or corrected
    std::shared_ptr<EdgeStats> snapshot; // the statistics then (after a correction: the live ones)
    std::shared_ptr<EdgeStats> live;     // the statistics the tree updates
    int max_edge = 62;
    OptimalTree(FlatTree t, std::shared_ptr<EdgeStats> stats);
    void replace(int node, const EdgeStats &st, int edge_no);   // Replace (:14-36)
    bool try_correct();                                        // TryCorrectTree (:38-93)
};

// CompressionOptimizer for one column (optimizer/compression_optimizer.hpp)
struct Optimizer {
    int dt;
    std::shared_ptr<EdgeStats> stats;
    std::unique_ptr<OptimalTree> opt;
    uint64_t parts = 0, total_bytes = 0;
    explicit Optimizer(int dtype) : dt(dtype), stats(std::make_shared<EdgeStats>(5)) {}
    // CompressData (:156-193): full update every 10th part (and the first), compress with the
    // optimal tree, fold its node ratios into the statistics, then try to correct the tree
    DevBuf compress_data(View part, bool *full_update, bool *corrected, cudaStream_t s);
};

}  // namespace gtsc
