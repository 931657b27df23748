// encodings.hpp -- host orchestration of each encoding (the reference's Encoding subclasses).
#pragma once

#include "common.cuh"

namespace gtsc {

// Encoding::Encode / Decode for one encoding type (compression/encoding.hpp:28-68).
// Encode returns [metadata, out1, (out2)].  Decode takes [metadata, in1, (in2)].
Parts encode(int enc, int dt, View in, cudaStream_t s);
DevBuf decode(int enc, int dt, const std::vector<View> &in, cudaStream_t s);

// the standalone UniqueEncoding (unique.cu)
Parts unique_encode(int dt, View in, cudaStream_t s);
DevBuf unique_decode(int dt, View meta, View data, cudaStream_t s);
// number of distinct values (bit patterns) of a column
uint64_t unique_count(int dt, View in, cudaStream_t s);

// number of child streams (GetNumberOfResults) and their data types (GetReturnTypes)
int n_results(int enc);
int return_type(int enc, int dt, int j);

// DataStatistics (util/statistics/cuda_array_statistics.hpp:24-34)
struct Stats {
    double min;
    double max;
    int32_t min_bit_cnt;
    int32_t precision;
    int32_t sorted;
    float rl_metric;
    double mean;
    uint64_t size;
};
// CudaArrayStatistics::GenerateStatistics (cuda_array_statistics.cu:141-179), one pass
Stats column_stats(int dt, View in, cudaStream_t s);

}  // namespace gtsc
