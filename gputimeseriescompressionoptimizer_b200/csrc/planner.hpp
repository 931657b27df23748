// planner.hpp -- plain exhaustive planner (CompressionOptimizer, optimizer/compression_optimizer.cpp)
#pragma once

#include "common.cuh"
#include "encodings.hpp"
#include "tree.hpp"

namespace gtsc {

struct PlanCounters {
    uint64_t encodes = 0;
    uint64_t stats_calls = 0;
};

// GetSampleDataForFullUpdateSize (compression_optimizer.cpp:148-154)
uint64_t sample_bytes(int dt, uint64_t bytes);
// FullStatisticsUpdate + the max-ratio pick of CompressData (compression_optimizer.cpp:88-182)
Tree plan_exhaustive(int dt, View sample, uint64_t *best_size, PlanCounters *counters, cudaStream_t s);
// one FullStatisticsUpdate candidate, Fix()ed: the tree, each node's compression ratio (pre-order)
// and the candidate's output size as the reference counts it
struct Candidate {
    Tree tree;
    std::vector<double> ratio;
    uint64_t size = 0;
};
// every candidate of FullStatisticsUpdate(sample, none, dt, 0), in the reference's order
std::vector<Candidate> plan_candidates(int dt, View sample, cudaStream_t s);
// CompressionOptimizer::OptimizeTree (compression_optimizer.cpp:16-36)
Tree optimize_tree(int dt, View data, uint64_t *best_size, cudaStream_t s);

}  // namespace gtsc
