// learned.hpp -- the learned tree planner: column features, a 32 -> 64 -> 64 -> K MLP (FP32) with
// hand-written training and inference kernels, and the planner that falls back to the exhaustive
// search when the network is not confident.  No counterpart in the reference, whose only planners
// are CompressionOptimizer::FullStatisticsUpdate / OptimizeTree (optimizer/compression_optimizer.cpp).
#pragma once

#include "common.cuh"
#include "tree.hpp"

#include <vector>

namespace gtsc {

constexpr int kFeatures = 32;
constexpr int kHidden = 64;
constexpr int kMaxClasses = 256;
constexpr uint32_t kFeatureSample = 10000;  // elements: the exhaustive planner's sample (GetSampleData...)
constexpr int kFeatureThreads = 1024;
constexpr uint32_t kFeatureSortCap = 16384;  // power of two >= kFeatureSample

struct FeatureColumn {
    const void *data;   // device column
    uint64_t n_total;   // elements in the whole column
    int dtype;
};
// features of every column's first min(n, kFeatureSample) elements into d_out[c * kFeatures + f]
void compute_features(const std::vector<FeatureColumn> &cols, float *d_out, cudaStream_t s);

// parameter layout (floats): W1[32x64] b1[64] W2[64x64] b2[64] W3[64xK] b3[K], W row-major (in x out)
inline size_t mlp_param_count(int K) { return (size_t)kFeatures * kHidden + kHidden + kHidden * kHidden + kHidden + (size_t)kHidden * K + K; }

class Planner {
public:
    int K = 0;
    std::vector<std::vector<int16_t>> classes;  // pre-order encoding lists
    std::vector<uint8_t> valid;                 // K x 6: class usable for a column of that data type
    std::vector<float> mu, sd;                  // feature normalisation (kFeatures each)
    DevBuf params, grads, adam_m, adam_v;       // device, mlp_param_count(K) floats each
    uint64_t adam_t = 0;

    Planner(const std::vector<std::vector<int16_t>> &cls, uint64_t seed);
    size_t n_params() const { return mlp_param_count(K); }
    void set_params(const float *h, cudaStream_t s);
    void get_params(float *h, cudaStream_t s) const;
    // mean loss and the gradient of the mean cross-entropy over rows (labels < 0 are skipped)
    float gradient(const float *d_x, const int32_t *h_labels, uint32_t n, float *h_grad, cudaStream_t s);
    // Adam over shuffled mini-batches; returns the mean loss of the last epoch
    float train(const float *d_x, const int32_t *h_labels, uint32_t n, int epochs, int batch, float lr, uint64_t seed,
                cudaStream_t s);
    // class and confidence (softmax probability renormalised over the classes valid for the dtype)
    void predict(const float *d_x, const int32_t *h_dtypes, uint32_t n, int32_t *h_class, float *h_conf,
                 cudaStream_t s);
    std::vector<uint8_t> save() const;
    static Planner *load(const void *bytes, uint64_t size);
    Tree class_tree(int c, int dtype) const;
};

}  // namespace gtsc
