// tree.hpp -- compression trees: the reference's CompressionTree / CompressionNode
// (tree/compression_tree.cpp, tree/compression_node.cpp) over the GPU encodings.
#pragma once

#include "common.cuh"
#include "encodings.hpp"

namespace gtsc {

// A tree is a pre-order list of (encoding, data type) nodes; each node is followed by its
// GetNumberOfResults() child subtrees and every leaf is `none` (a Fix()ed tree).
struct Tree {
    std::vector<int16_t> enc, dt;
    int size() const { return (int)enc.size(); }
};

Tree tree_from_nodes(const int16_t *pairs, int n_nodes);  // validates the shape
void tree_to_nodes(const Tree &t, int16_t *pairs);
// PathGenerator::GenerateTree (optimizer/path_generator.cpp:70-91): data types follow GetReturnTypes
Tree tree_from_path(const int16_t *encs, int n, int dtype);
// CompressionNode::Fix (tree/compression_node.cpp:209-223) of a single-node tree
Tree leaf_tree(int enc, int dtype);

// CompressionTree::Compress (tree/compression_tree.cpp:98-103): the serialized blob; `ratios`, when
// given, receives each node's compression ratio in pre-order (CompressionNode::Compress)
DevBuf tree_compress(const Tree &t, View in, cudaStream_t s, std::vector<double> *ratios = nullptr);
// Encoding::GetCompressionRatio (compression/encoding.hpp:78-84)
double compression_ratio(uint64_t in, uint64_t out);
// CompressionTree::Decompress (tree/compression_tree.cpp:105-155); *dtype = root data type
DevBuf tree_decompress(View blob, int *dtype, cudaStream_t s);
// CompressionNode::PredictCompressionSize (tree/compression_node.cpp:163-177)
uint64_t tree_predict_size(const Tree &t, View in, cudaStream_t s);

// GetMetadataSize of one encoding for `in` of type dt (the predictors of compression/*/ *.hpp)
uint64_t predicted_metadata_size(int enc, int dt, View in, cudaStream_t s);

}  // namespace gtsc
