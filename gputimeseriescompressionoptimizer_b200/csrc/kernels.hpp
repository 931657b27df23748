// kernels.hpp -- host launchers of the device kernels (one declaration per kernel family).
#pragma once

#include "common.cuh"

namespace gtsc {

// ---- min / max (minmax.cu) ---------------------------------------------------------------
// Folds the elements of in[0..n) into *acc (which the caller zeroes first) in order `o`.
// Floating NaNs are skipped.  `in` must be aligned to the element size.
void launch_minmax(const uint8_t *in, uint64_t n, int es, Order o, MinMaxAcc *acc, cudaStream_t s);
// Host-side decode of an accumulator (raw bits of min and max); `first` = bits of element 0,
// used when every element was NaN.  Returns false when nothing was seen.
bool minmax_result(const MinMaxAcc &acc, int es, Order o, uint64_t *mn, uint64_t *mx);

// ---- AFL fixed-width packing (afl.cu) ------------------------------------------------------
// Packs in[0..n) (elements of es bytes) at b bits each into the little-endian LSB-first
// bitstream out[0..out_bytes).  `in` and `out` 16-byte aligned.
void launch_afl_pack(const uint8_t *in, uint64_t n, int es, int b, uint8_t *out, uint64_t out_bytes,
                     cudaStream_t s);
// Unpacks n values of b bits starting at stream byte 0 of `stream` (any alignment) into out.
void launch_afl_unpack(const uint8_t *stream, uint64_t stream_bytes, uint64_t n, int es, int b,
                       uint8_t *out, cudaStream_t s);

}  // namespace gtsc
