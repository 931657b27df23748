// encodings.hpp -- host orchestration of each encoding (the reference's Encoding subclasses).
#pragma once

#include "common.cuh"

namespace gtsc {

// Encoding::Encode / Decode for one encoding type (compression/encoding.hpp:28-68).
// Encode returns [metadata, out1, (out2)].  Decode takes [metadata, in1, (in2)].
Parts encode(int enc, int dt, View in, cudaStream_t s);
DevBuf decode(int enc, int dt, const std::vector<View> &in, cudaStream_t s);

// number of child streams (GetNumberOfResults) and their data types (GetReturnTypes)
int n_results(int enc);
int return_type(int enc, int dt, int j);

}  // namespace gtsc
