/*
 * oracle.h -- CPU restatement of the reference's lightweight column-compression path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or calls this code.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs use it,
 * and only as the checker or as the timed CPU baseline.
 *
 * Every function restates one reference function (cited file:line, paths inside the reference
 * project).  Pins:
 *   - AFL is cross-checked against the reference's own afl_gpu.cu host path, compiled from its
 *     sources into oracle/_ref/ (see oracle/Makefile, target `ref`).
 *   - BITLEN / ALT_BITLEN, _getFloatPrecision, Sorted, RlMetric, Mean, stencil, split/merge, unique
 *     and tree round-trips are pinned by the known-answer tests restated in tests/.
 *   - The remaining byte layouts (delta, scale, RLE, dict/unique, const, patch, floatToInt, none,
 *     GFC, serialized tree) have no golden vectors in the reference: they follow the reference
 *     source line by line and are "parity pinned by KAT + restatement", not by reference output.
 *
 * Data types use the codes below; the reference's DataType numeric values live in a submodule that
 * is not available, so header bytes 2-3 of a serialized node use this mapping.
 */
#ifndef GTSC_ORACLE_H_
#define GTSC_ORACLE_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum or_dtype { OR_CHAR = 0, OR_SHORT = 1, OR_INT = 2, OR_TIME = 3, OR_FLOAT = 4, OR_DOUBLE = 5 };

/* compression/encoding_type.hpp:17-30 */
enum or_enc {
    OR_DELTA = 0, OR_AFL = 1, OR_SCALE = 2, OR_RLE = 3, OR_DICT = 4, OR_UNIQUE = 5,
    OR_PATCH = 6, OR_NONE = 7, OR_FLOAT2INT = 8, OR_CONST = 9, OR_GFC = 10,
    /* PatchEncodingFactory(dt, PatchType::outside) (patch_encoding_factory.hpp:47-55): encoded by
     * OutsidePatchEncoding, serialised and decoded as patch (6) */
    OR_PATCH_OUTSIDE = 11
};

enum or_status {
    OR_OK = 0, OR_ERR_ARG = -1, OR_ERR_TYPE = -2, OR_ERR_CAP = -3, OR_ERR_FORMAT = -4,
    OR_ERR_UNSUPPORTED = -5
};

int or_dtype_size(int dtype);

/* core/cuda_macros.cuh:168-205 */
int or_bitlen(int dtype, int64_t min, int64_t max);
int or_alt_bitlen(int v);

/*
 * Encoding::Encode (compression/encoding.hpp:28-47): writes up to three output buffers
 * (out[0] = metadata).  Each buffer must hold `cap` bytes.  Returns OR_OK or an error.
 */
int or_encode(int enc, int dtype, const uint8_t *in, uint64_t in_bytes,
              uint8_t *out0, uint8_t *out1, uint8_t *out2, uint64_t cap,
              uint64_t out_bytes[3], int *n_out);

/*
 * The packed AFL layouts by bit position (afl_gpu.cu:5-65, 197-222): omega 1 (FL) or 32
 * (aligned).  or_afl_words = words of n elements at b bits; or_afl_pack writes them (zero
 * filled); or_afl_values reads element idx[t] (t when idx is NULL) for t < n.
 */
uint64_t or_afl_words(int omega, int dtype, int b, uint64_t n);
int or_afl_pack(int omega, int dtype, int b, const uint8_t *in, uint64_t n, uint8_t *out, uint64_t words);
int or_afl_values(int omega, int dtype, int b, const uint8_t *comp, uint64_t words, const uint64_t *idx,
                  uint64_t n, uint8_t *out);

/* Encoding::Decode (compression/encoding.hpp:49-68). */
int or_decode(int enc, int dtype,
              const uint8_t *in0, uint64_t b0, const uint8_t *in1, uint64_t b1,
              const uint8_t *in2, uint64_t b2,
              uint8_t *out, uint64_t cap, uint64_t *out_bytes);

/* DataStatistics (util/statistics/cuda_array_statistics.hpp:24-34). */
typedef struct {
    double min;
    double max;
    int32_t min_bit_cnt;
    int32_t precision;
    int32_t sorted;
    float rl_metric;
    double mean;
    uint64_t size;
} or_stats_t;

/* CudaArrayStatistics::GenerateStatistics (util/statistics/cuda_array_statistics.cu:141-179). */
int or_stats(int dtype, const uint8_t *in, uint64_t in_bytes, or_stats_t *out);
/* CudaArrayStatistics::RlMetric<T,N> (cuda_array_statistics.cu:97-132), N in 2..6. */
float or_rl_metric(int dtype, const uint8_t *in, uint64_t in_bytes, int N);
/* _getFloatPrecision (cuda_array_statistics.cu:37-44). */
int or_float_precision(float x);

/* Stencil::pack / unpack (util/stencil/stencil.cu:14-96).  stencil: one int32 0/1 per element. */
uint64_t or_stencil_pack(const int32_t *stencil, uint64_t n, uint8_t *out);
int64_t or_stencil_unpack(const uint8_t *packed, uint64_t bytes, int32_t *out, uint64_t cap);

/*
 * Compression trees are passed as pre-order node lists: node k = (nodes[2k] = encoding type,
 * nodes[2k+1] = data type); a node is followed by its GetNumberOfResults() child subtrees and every
 * leaf is `none` (a Fix()ed tree, tree/compression_node.cpp:209-223).
 *
 * or_tree_from_path: PathGenerator::GenerateTree (optimizer/path_generator.cpp:70-91) -- data types
 * follow each encoding's GetReturnTypes.  Returns the node count or an error.
 */
int or_tree_from_path(const int16_t *encs, int n_encs, int dtype, int16_t *nodes, int cap);
/* CompressionTree::Compress (tree/compression_tree.cpp:98-103, tree/compression_node.cpp:84-138) */
int or_tree_compress(const int16_t *nodes, int n_nodes,
                     const uint8_t *in, uint64_t in_bytes,
                     uint8_t *out, uint64_t cap, uint64_t *out_bytes);
/* CompressionTree::Decompress (tree/compression_tree.cpp:105-155) */
int or_tree_decompress(const uint8_t *blob, uint64_t blob_bytes,
                       uint8_t *out, uint64_t cap, uint64_t *out_bytes, int *dtype);
/* CompressionNode::PredictCompressionSize (tree/compression_node.cpp:163-177). */
int or_tree_predict_size(const int16_t *nodes, int n_nodes,
                         const uint8_t *in, uint64_t in_bytes, uint64_t *size);

/*
 * Plain exhaustive planner: CompressionOptimizer::FullStatisticsUpdate + the max-ratio pick of
 * CompressData phase 1 (optimizer/compression_optimizer.cpp:88-140, 156-182), evaluated on the
 * given sample.  Writes the chosen Fix()ed tree and its candidate size.
 */
int or_plan_exhaustive(int dtype, const uint8_t *in, uint64_t in_bytes,
                       int16_t *nodes_out, int cap, int *n_nodes, uint64_t *best_size);
/* CompressionOptimizer::OptimizeTree (optimizer/compression_optimizer.cpp:16-36). */
int or_optimize_tree(int dtype, const uint8_t *in, uint64_t in_bytes,
                     int16_t *nodes_out, int cap, int *n_nodes, uint64_t *best_size);
/* GetSampleDataForFullUpdateSize (compression_optimizer.cpp:148-154): bytes of the planner sample */
uint64_t or_sample_bytes(int dtype, uint64_t in_bytes);

#ifdef __cplusplus
}
#endif
#endif
