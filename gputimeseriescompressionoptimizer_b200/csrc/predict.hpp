// predict.hpp -- the encodings' size predictors (Encoding::GetMetadataSize / GetCompressedSize).
#pragma once

#include "common.cuh"

namespace gtsc {

struct SizePrediction {
    uint64_t meta;   // GetMetadataSize
    uint64_t data;   // GetCompressedSize: the data outputs together
};
SizePrediction predict_sizes(int enc, int dt, View in, cudaStream_t s);

}  // namespace gtsc
