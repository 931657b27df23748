/*
 * gtsc.h -- C ABI of the B200 column-compression library (libgtsc.so).
 *
 * Every entry point takes plain pointers and sizes, returns a gtsc_status, and runs its GPU work on
 * the given CUDA stream (a cudaStream_t passed as void*; NULL = the legacy default stream).  Device
 * buffers returned through gtsc_buffer are allocated by the library with stream-ordered
 * cudaMallocAsync and belong to the caller, who releases them with gtsc_free.  Nothing here exits
 * the process: CUDA and format errors come back as status codes (gtsc_last_error() has the text).
 *
 * Encoding and data-type codes follow the reference's enums (compression/encoding_type.hpp:17-30;
 * the DataType values live in a submodule that is not available, so the codes below are this
 * library's own and are what it writes into serialized node headers).
 */
#ifndef GTSC_H_
#define GTSC_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gtsc_status;
enum {
    GTSC_OK = 0,
    GTSC_ERR_ARG = -1,          /* bad argument (null pointer, unknown code)                */
    GTSC_ERR_TYPE = -2,         /* encoding not defined for this data type                  */
    GTSC_ERR_CAPACITY = -3,     /* output buffer too small / size above a stated maximum    */
    GTSC_ERR_FORMAT = -4,       /* corrupt or truncated compressed input                    */
    GTSC_ERR_UNSUPPORTED = -5,  /* reference entry point without a GPU counterpart          */
    GTSC_ERR_CUDA = -6,         /* CUDA runtime error                                       */
    GTSC_ERR_TIMEOUT = -7,      /* a bounded device-side wait gave up                       */
    GTSC_ERR_NO_DEVICE = -8     /* no CUDA device                                           */
};

/* DataType (reference: modules/data, unavailable) -- this library's codes */
enum { GTSC_CHAR = 0, GTSC_SHORT = 1, GTSC_INT = 2, GTSC_TIME = 3, GTSC_FLOAT = 4, GTSC_DOUBLE = 5 };

/* EncodingType -- compression/encoding_type.hpp:17-30 */
enum {
    GTSC_DELTA = 0, GTSC_AFL = 1, GTSC_SCALE = 2, GTSC_RLE = 3, GTSC_DICT = 4, GTSC_UNIQUE = 5,
    GTSC_PATCH = 6, GTSC_NONE = 7, GTSC_FLOAT_TO_INT = 8, GTSC_CONST = 9, GTSC_GFC = 10,
    /* The outside variant of the patch encoding: PatchEncodingFactory<T>(dt, PatchType::outside)
     * (compression/patch/patch_encoding_factory.hpp:47-55) building an OutsidePatchEncoding
     * (outside_patch_encoding.cu:22-60).  GTSC_PATCH is the lower variant, the one
     * DefaultEncodingFactory uses (default_encoding_factory.hpp:48-60).  Accepted by gtsc_encode /
     * gtsc_decode and in tree node lists; a serialised tree records it as GTSC_PATCH (6), as the
     * reference does, and both variants decode alike. */
    GTSC_PATCH_OUTSIDE = 11
};

typedef struct {
    void *ptr;        /* device pointer (may be NULL when bytes == 0) */
    uint64_t bytes;
} gtsc_buffer;

/* ------------------------------------------------------------------ runtime / memory */

/* Text of the last error raised on the calling thread ("" when none). */
const char *gtsc_last_error(void);
/* Library version string. */
const char *gtsc_version(void);
/* Size in bytes of one element of `dtype` (0 for an unknown code).  GetDataTypeSize. */
int32_t gtsc_dtype_size(int32_t dtype);
/* Stream-ordered device allocation / release (cudaMallocAsync / cudaFreeAsync). */
gtsc_status gtsc_malloc(void **d_ptr, uint64_t bytes, void *stream);
gtsc_status gtsc_free(void *d_ptr, void *stream);
/* Copies; `kind` 1 = host->device, 2 = device->host, 3 = device->device (cudaMemcpyKind). */
gtsc_status gtsc_memcpy(void *dst, const void *src, uint64_t bytes, int32_t kind, void *stream);
/* The same copy, never synchronising (host memory must be pinned for it to overlap). */
gtsc_status gtsc_memcpy_async(void *dst, const void *src, uint64_t bytes, int32_t kind, void *stream);
gtsc_status gtsc_stream_synchronize(void *stream);
/* A non-blocking CUDA stream (the batched steps need one they can capture on). */
gtsc_status gtsc_stream_create(void **stream);
gtsc_status gtsc_stream_destroy(void *stream);

/* ------------------------------------------------------------------ encodings */

/*
 * Encoding::Encode(SharedCudaPtr<char> data, DataType) (compression/encoding.hpp:28-47).
 * Writes out[0] = metadata, out[1..n_out-1] = encoded streams, byte-identical to the reference
 * encoder for the same input (bytes the reference leaves uninitialised -- AFL metadata bytes 2-3,
 * unused dictionary slots, dictionary code bits past the last value -- are written as 0; the
 * dictionary's top-4 ties are ordered by value).  Synchronises the
 * stream once to learn the data-dependent output sizes, as the reference does.
 */
gtsc_status gtsc_encode(int32_t encoding, int32_t dtype, const void *d_in, uint64_t in_bytes,
                        gtsc_buffer out[3], uint32_t *n_out, void *stream);

/* Encoding::Decode(SharedCudaPtrVector<char>, DataType) (compression/encoding.hpp:49-68). */
gtsc_status gtsc_decode(int32_t encoding, int32_t dtype, const gtsc_buffer in[3], uint32_t n_in,
                        gtsc_buffer *out, void *stream);

/* DataStatistics (util/statistics/cuda_array_statistics.hpp:24-34) */
typedef struct {
    double min;
    double max;
    int32_t min_bit_cnt;
    int32_t precision;
    int32_t sorted;
    float rl_metric;
    double mean;
    uint64_t size;
} gtsc_data_statistics;

/*
 * CudaArrayStatistics::GenerateStatistics (util/statistics/cuda_array_statistics.cu:141-179):
 * min, max, precision, sorted, RlMetric<T,2> and mean of a column in one pass over the data.
 */
gtsc_status gtsc_stats(int32_t dtype, const void *d_in, uint64_t in_bytes, gtsc_data_statistics *out,
                       void *stream);

/* ------------------------------------------------------------------ compression trees */

/*
 * Trees are pre-order node lists: node k = (nodes[2k] = EncodingType, nodes[2k+1] = DataType), each
 * node followed by its GetNumberOfResults() child subtrees, every leaf `none` (a Fix()ed tree,
 * tree/compression_node.cpp:209-223).
 *
 * PathGenerator::GenerateTree (optimizer/path_generator.cpp:70-91): builds the node list of a path
 * of encoding types, children typed by GetReturnTypes.  Returns GTSC_ERR_CAPACITY when more than
 * `cap` nodes would be written.
 */
gtsc_status gtsc_tree_from_path(const int16_t *encodings, int32_t n_encodings, int32_t dtype,
                                int16_t *nodes_out, int32_t cap, int32_t *n_nodes);

/* CompressionTree::Compress (tree/compression_tree.cpp:98-103): serialized blob of the column. */
gtsc_status gtsc_tree_compress(const int16_t *nodes, int32_t n_nodes, const void *d_in, uint64_t in_bytes,
                               gtsc_buffer *blob, void *stream);

/* CompressionTree::Decompress (tree/compression_tree.cpp:105-155); *dtype = the root's data type. */
gtsc_status gtsc_tree_decompress(const void *d_blob, uint64_t blob_bytes, gtsc_buffer *out, int32_t *dtype,
                                 void *stream);

/* CompressionTree::GetPredictedSizeAfterCompression (tree/compression_tree.cpp:157-160). */
gtsc_status gtsc_tree_predict_size(const int16_t *nodes, int32_t n_nodes, const void *d_in, uint64_t in_bytes,
                                   uint64_t *size, void *stream);

/* ------------------------------------------------------------------ planners */

/*
 * The plain exhaustive planner: CompressionOptimizer::FullStatisticsUpdate on `d_sample` and the
 * max-compression-ratio pick of CompressData (optimizer/compression_optimizer.cpp:88-182).  Writes the
 * chosen Fix()ed tree and its candidate size (as the reference counts it).
 */
gtsc_status gtsc_plan_exhaustive(int32_t dtype, const void *d_sample, uint64_t sample_bytes, int16_t *nodes_out,
                                 int32_t cap, int32_t *n_nodes, uint64_t *candidate_size, void *stream);

/* CompressionOptimizer::OptimizeTree (optimizer/compression_optimizer.cpp:16-36): best of 30 paths. */
gtsc_status gtsc_optimize_tree(int32_t dtype, const void *d_in, uint64_t in_bytes, int16_t *nodes_out,
                               int32_t cap, int32_t *n_nodes, uint64_t *predicted_size, void *stream);

/* GetSampleDataForFullUpdateSize (optimizer/compression_optimizer.cpp:148-154). */
uint64_t gtsc_sample_bytes(int32_t dtype, uint64_t in_bytes);

/* ------------------------------------------------------------------ batched columns */

/*
 * Compresses many columns, each with its own tree, in a fixed sequence of batched launches that is
 * recorded once as a CUDA graph.  It replaces the per-column task loop of the reference
 * (ParallelTSCompressor::Compress, parallel_ts_compressor.cpp:39-63, one CompressionTask per column,
 * optimizer/compression_task.cpp:42-77) for columns whose trees are known.  Framed output: uint64
 * column count C, a directory of C uint64 blob byte counts (the size_t length the reference writes
 * before each chunk, compression_task.cpp:35-40, gathered in front so decode finds every column at
 * once), then the C blobs of CompressionTree::Compress back to back.  All column and output
 * pointers must be 16-byte aligned.
 */
typedef struct gtsc_batch gtsc_batch;
typedef struct {
    const void *d_data;   /* device column */
    uint64_t bytes;
    int32_t dtype;
    int32_t reserved;
} gtsc_column;

/* nodes: the columns' node lists concatenated; node_counts[c] = nodes of column c.  stream must
 * not be the legacy default stream (steps are captured on it). */
gtsc_status gtsc_batch_create(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                              const int32_t *node_counts, gtsc_batch **out, void *stream);
/* new device pointers for the columns (same sizes), used by the next compress */
gtsc_status gtsc_batch_set_inputs(gtsc_batch *b, const void *const *d_inputs, void *stream);
/* one compress step (asynchronous): framed output in the batch's device buffer */
gtsc_status gtsc_batch_compress(gtsc_batch *b, void *stream);
/* the framed output of the last compress and its byte count (synchronises) */
gtsc_status gtsc_batch_output(gtsc_batch *b, const void **d_framed, uint64_t *bytes, void *stream);
/* blob bytes of every column in the last compress (synchronises) */
gtsc_status gtsc_batch_blob_sizes(gtsc_batch *b, uint64_t *sizes, void *stream);
/* one decompress step (asynchronous) of a framed buffer made by any compress step of this batch */
gtsc_status gtsc_batch_decompress(gtsc_batch *b, const void *d_framed, uint64_t framed_bytes,
                                  void *const *d_outputs, void *stream);
/* status of the steps run so far (synchronises): a device-side format, capacity or timeout error */
gtsc_status gtsc_batch_status(gtsc_batch *b, void *stream);
/* kernel launches in one step (compress != 0: compress step) */
int32_t gtsc_batch_launches(gtsc_batch *b, int32_t compress);
/*
 * The schedule later steps replay (both are recorded at creation): GTSC_SCHEDULE_LEVELS = one launch
 * per (tree level, pass kind) over all columns; GTSC_SCHEDULE_PERSISTENT = one persistent launch per
 * step whose blocks pull (pass, tile) work from a device queue, each column's levels waiting only for
 * that column's earlier levels (then a compress step is 6 launches and a decompress step 4).  Both
 * give the same bytes.  The default is the levels; gtsc_batch_autotune picks by measurement.
 * No counterpart in the reference (it compresses one column at a time).
 */
enum { GTSC_SCHEDULE_LEVELS = 0, GTSC_SCHEDULE_PERSISTENT = 1 };
gtsc_status gtsc_batch_set_schedule(gtsc_batch *b, int32_t schedule);
int32_t gtsc_batch_schedule(gtsc_batch *b);
/*
 * Launch parameters of a batch, and the autotuner that chooses them (no counterpart in the
 * reference, whose launch configuration is fixed, core/execution_policy.hpp:14-49).  Tiles are
 * values per block tile.  Defaults: min/max tile 8192 with 16 values per thread, histogram tile
 * 32768, level schedule for both steps.
 */
typedef struct {
    uint32_t minmax_tile;               /* 1024 .. 16384, a multiple of 256 x the values per thread */
    uint32_t minmax_values_per_thread;  /* consecutive values a thread loads per round: 1, 2, 4, 8, 16 */
    uint32_t hist_tile;                 /* dict / const histogram: a multiple of 256, at most 32768 */
    int32_t schedule_compress;          /* GTSC_SCHEDULE_* */
    int32_t schedule_decompress;
    /* filled by gtsc_batch_autotune: step times (ms) with the default and with the chosen
     * parameters, candidates timed, seconds spent */
    float ms_default_compress, ms_default_decompress, ms_tuned_compress, ms_tuned_decompress;
    int32_t candidates;
    float seconds;
} gtsc_batch_tuning;
/* gtsc_batch_create with explicit launch parameters (NULL: the defaults) */
gtsc_status gtsc_batch_create_tuned(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                                    const int32_t *node_counts, const gtsc_batch_tuning *tuning, gtsc_batch **out,
                                    void *stream);
gtsc_status gtsc_batch_get_tuning(gtsc_batch *b, gtsc_batch_tuning *tuning);
/*
 * Times candidate parameters on the batch's own columns and trees with CUDA events: the schedule of
 * each step; then the min/max tile (1K .. 16K) x values per thread (1 .. 16) on the min/max
 * launches; then the histogram tile (8K .. 32K) on the histogram and top-k launches (a rebuild
 * each); a candidate is kept when it is at least 2 % faster.  The batch keeps the best parameters
 * (its device buffers, the framed output included, may move: call gtsc_batch_output again).
 * Synchronises; a few seconds for hundreds of columns.  *report may be NULL.
 */
gtsc_status gtsc_batch_autotune(gtsc_batch *b, gtsc_batch_tuning *report, void *stream);
/*
 * One step run launch by launch with CUDA events between the launches (not the graph): per launch
 * its pass kind (ops[i] >= 0, or -1 stream setup, -2 scratch zeroing, -3/-4/-5 frame sizes / layout
 * / copy, -6 frame parse, -7 the persistent launch of every pass), its time in ms, the bytes it must read and write at least (its input and
 * output streams) and its blocks.  Writes at most cap entries and the count to *n.  Synchronises.
 * No counterpart in the reference (its per-column calls are timed one by one).
 */
gtsc_status gtsc_batch_profile(gtsc_batch *b, int32_t compress, int32_t *ops, float *ms, uint64_t *bytes,
                               uint64_t *blocks, int32_t cap, int32_t *n, void *stream);
gtsc_status gtsc_batch_destroy(gtsc_batch *b);

/* ------------------------------------------------------------------ column-chunk pipeline */

/*
 * Column chunks from host memory to host framed output: ParallelTSCompressor::Compress's chunk loop
 * (parallel_ts_compressor.cpp:39-63, a CompressionTask per column chunk writing size_t len + blob,
 * optimizer/compression_task.cpp:35-77) on the batched engine.  The columns are split into `groups`
 * of about equal bytes, each with its own batch engine and stream, so that one group's host <->
 * device copies overlap the others' compression.  The pipeline owns the device copies of the
 * columns (cols[].d_data is ignored; bytes and dtype fix the chunk shape).
 */
typedef struct gtsc_pipeline gtsc_pipeline;
gtsc_status gtsc_pipeline_create(const gtsc_column *cols, uint32_t n_cols, const int16_t *nodes,
                                 const int32_t *node_counts, int32_t groups, gtsc_pipeline **out);
int32_t gtsc_pipeline_groups(gtsc_pipeline *p);
/* The columns of group g in the order of its framed output (ascending column index). */
gtsc_status gtsc_pipeline_group_columns(gtsc_pipeline *p, int32_t g, int32_t *cols, int32_t cap, int32_t *n);
/* One chunk: host_cols[c] (pinned for overlap) -> host_framed = every group's framed output
 * (column count, blob sizes, blobs) back to back, group_bytes[g] their sizes.  Synchronises. */
gtsc_status gtsc_pipeline_compress_host(gtsc_pipeline *p, const void *const *host_cols, void *host_framed,
                                        uint64_t cap, uint64_t *group_bytes);
/* The same chunk plus, per group right after its framed output is read back, the device decode
 * of that output into the per-column output buffers (a verified round trip of the chunk). */
gtsc_status gtsc_pipeline_roundtrip_host(gtsc_pipeline *p, const void *const *host_cols, void *host_framed,
                                         uint64_t cap, uint64_t *group_bytes);
/* Decodes the last compressed chunk on the device (every group's step in flight together) into
 * the pipeline's per-column output buffers; the first failing status is returned. */
gtsc_status gtsc_pipeline_decompress(gtsc_pipeline *p);
/* Device buffers of column c: its last input chunk and its last decoded output. */
gtsc_status gtsc_pipeline_column(gtsc_pipeline *p, int32_t c, const void **d_input, const void **d_output);
gtsc_status gtsc_pipeline_destroy(gtsc_pipeline *p);

/* ------------------------------------------------------------------ learned planner */

/*
 * A small MLP over column features proposes the compression tree; the exhaustive planner above is
 * its fallback.  No counterpart in the reference (its planners are FullStatisticsUpdate and
 * OptimizeTree, optimizer/compression_optimizer.cpp:16-140); it stands beside gtsc_plan_exhaustive
 * and returns trees in the same node-list form.
 *
 * Features: 32 floats per column from its first min(n, 10000) elements (the exhaustive planner's
 * sample, GetSampleDataForFullUpdateSize): data-type one-hot, size, NaN / inf share, sortedness,
 * runs, distinct values and the largest multiplicities, value / delta / second-delta bit widths,
 * float precision and floatToInt feasibility.  d_features: device, n_cols x 32, row-major.
 */
#define GTSC_PLANNER_FEATURES 32
typedef struct gtsc_planner gtsc_planner;
gtsc_status gtsc_planner_features(const gtsc_column *cols, uint32_t n_cols, float *d_features, void *stream);
/* A new network (He-uniform from `seed`) over n_classes tree classes: class c is the pre-order
 * encoding list class_encs[off_c .. off_c + class_lens[c]) (the lists concatenated). */
gtsc_status gtsc_planner_create(const int16_t *class_encs, const int32_t *class_lens, int32_t n_classes,
                                uint64_t seed, gtsc_planner **out);
/* Serialized model ("GTSCMLP1": shape, normalisation, parameters, class table). */
gtsc_status gtsc_planner_load(const void *model, uint64_t bytes, gtsc_planner **out);
gtsc_status gtsc_planner_save(gtsc_planner *p, void *buf, uint64_t cap, uint64_t *bytes);
gtsc_status gtsc_planner_destroy(gtsc_planner *p);
int32_t gtsc_planner_classes(gtsc_planner *p);
/* parameters: W1[32x64] b1[64] W2[64x64] b2[64] W3[64xK] b3[K] (W row-major, in x out) */
uint64_t gtsc_planner_param_count(gtsc_planner *p);
gtsc_status gtsc_planner_get_params(gtsc_planner *p, float *params, float *mu, float *sd);
gtsc_status gtsc_planner_set_params(gtsc_planner *p, const float *params, const float *mu, const float *sd);
/* valid[c * 6 + dtype] = 1 when class c can encode a column of that data type */
gtsc_status gtsc_planner_valid(gtsc_planner *p, uint8_t *valid);
/* Mean cross-entropy over the rows (label < 0: skipped) and its gradient w.r.t. the parameters,
 * by the library's forward and backward kernels (FP32, fixed summation order). */
gtsc_status gtsc_planner_gradient(gtsc_planner *p, const float *d_features, const int32_t *labels, uint32_t n_rows,
                                  float *grad, float *loss, void *stream);
/* Adam over shuffled mini-batches on the device; sets the feature normalisation from the rows. */
gtsc_status gtsc_planner_train(gtsc_planner *p, const float *d_features, const int32_t *labels, uint32_t n_rows,
                               int32_t epochs, int32_t batch, float lr, uint64_t seed, float *final_loss,
                               void *stream);
/* Most probable valid class per row and its probability among the classes valid for the dtype. */
gtsc_status gtsc_planner_predict(gtsc_planner *p, const float *d_features, const int32_t *dtypes, uint32_t n_rows,
                                 int32_t *classes, float *confidence, void *stream);
/* Trees for many columns: the network's class where its confidence >= min_confidence, else the
 * exhaustive planner on the column's sample (fallback[c] = 1).  Node lists are written back to
 * back into nodes_out (pairs), node_counts[c] nodes for column c. */
gtsc_status gtsc_plan_learned(gtsc_planner *p, const gtsc_column *cols, uint32_t n_cols, float min_confidence,
                              int16_t *nodes_out, int32_t nodes_cap, int32_t *node_counts, int32_t *fallback,
                              void *stream);

/* ------------------------------------------------------------------ kernel-level entry points */

/*
 * run_afl_compress_gpu<T,1> (compression/afl/afl_gpu.cu:67-73): packs n elements of an integer
 * `dtype` at bit_length bits into d_out (out_bytes = ceil(n*b / W) * sizeof(T), W = 8*sizeof(T)),
 * the FL layout of AflEncoding.  Asynchronous; d_data and d_out 16-byte aligned.
 */
gtsc_status gtsc_afl_compress_gpu(int32_t dtype, uint32_t bit_length, const void *d_data, uint64_t n,
                                  void *d_out, uint64_t out_bytes, void *stream);
/* run_afl_decompress_gpu<T,1> (afl_gpu.cu:75-81): unpacks n values; d_comp may be unaligned. */
gtsc_status gtsc_afl_decompress_gpu(int32_t dtype, uint32_t bit_length, const void *d_comp,
                                    uint64_t comp_bytes, void *d_out, uint64_t n, void *stream);

/*
 * Encoding::GetMetadataSize / GetCompressedSize (compression/encoding.hpp:74-76; the per-encoding
 * predictors, e.g. rle_encode.cu:64-97, dict_encoding.cu:132-161, afl_encoding.cu:281-343,
 * unique_encoding.cu:306-326): *metadata_bytes = the size of out[0], *compressed_bytes = the sizes
 * of the data outputs together, computed by counting passes without encoding.  Exact for none,
 * delta, scale, rle, dict, const, integer afl and unique; patch and floatToInt predict the input
 * size, gfc 0 data bytes and float afl 9 metadata bytes, as the reference's predictors do.
 * Synchronises the stream.
 */
gtsc_status gtsc_predict_sizes(int32_t encoding, int32_t dtype, const void *d_in, uint64_t in_bytes,
                               uint64_t *metadata_bytes, uint64_t *compressed_bytes, void *stream);

/*
 * run_afl_compress_gpu<T,32> / run_afl_decompress_gpu<T,32> (compression/afl/afl_gpu.cu:67-81, the
 * aligned layout instantiated at afl_gpu.cu:263-265): blocks of 32*W values (W = element bits),
 * value j of lane l of a block at element 32j + l, lane l's packed words at 32k + l.  The packed
 * stream takes gtsc_afl32_bytes(dtype, b, n) bytes (whole blocks; holes in the last one are 0).
 * Integer types; element-aligned pointers.
 */
uint64_t gtsc_afl32_bytes(int32_t dtype, uint32_t bit_length, uint64_t n);
gtsc_status gtsc_afl32_compress_gpu(int32_t dtype, uint32_t bit_length, const void *d_data, uint64_t n, void *d_out,
                                    uint64_t out_bytes, void *stream);
gtsc_status gtsc_afl32_decompress_gpu(int32_t dtype, uint32_t bit_length, const void *d_comp, uint64_t comp_bytes,
                                      void *d_out, uint64_t n, void *stream);
/*
 * Random-access decode, run_afl_decompress_value_gpu<T,omega> (afl_gpu.cu:83-121, 197-222):
 * out[t] = element (d_index ? d_index[t] : t) of an FL (omega 1, AflEncoding's layout) or aligned
 * (omega 32) packed stream, for t < n; each element is decoded on its own.
 */
gtsc_status gtsc_afl_values_gpu(int32_t dtype, uint32_t bit_length, int32_t omega, const void *d_comp,
                                uint64_t comp_bytes, const uint64_t *d_index, uint64_t n, void *d_out, void *stream);

/*
 * Online tree maintenance: CompressionOptimizer::CompressData (optimizer/compression_optimizer.cpp
 * 142-193) for one column.  Each call compresses one part (a chunk of the column) and returns its
 * serialized tree blob.  The first part and every 10th after run a full statistics update:
 * every FullStatisticsUpdate candidate on the part's first 10 000 elements is folded into the edge
 * statistics (CompressionTree::UpdateStatistics, tree/compression_tree.cpp:232-240) and the best
 * becomes the optimal tree.  Every part is compressed with the optimal tree, its node ratios folded
 * in, and the tree corrected (OptimalTree::TryCorrectTree, optimizer/optimal_tree.cpp:38-93).
 * *full_update / *corrected (optional) report what this call did.  The blob decodes with
 * gtsc_tree_decompress.
 */
typedef struct gtsc_optimizer gtsc_optimizer;
gtsc_status gtsc_optimizer_create(int32_t dtype, gtsc_optimizer **out);
gtsc_status gtsc_optimizer_compress(gtsc_optimizer *o, const void *d_in, uint64_t in_bytes, gtsc_buffer *blob,
                                    int32_t *full_update, int32_t *corrected, void *stream);
/* GetOptimalTree()->GetTree(): pre-order (encoding, data type) pairs and each node's last ratio */
gtsc_status gtsc_optimizer_tree(const gtsc_optimizer *o, int16_t *nodes_out, double *ratios_out, int32_t cap,
                                int32_t *n_nodes);
/* GetStatistics(): the statistics object the optimizer updates (owned by it; valid until destroy) */
typedef struct gtsc_edge_stats gtsc_edge_stats;
gtsc_status gtsc_optimizer_statistics(gtsc_optimizer *o, gtsc_edge_stats **stats);
gtsc_status gtsc_optimizer_destroy(gtsc_optimizer *o);

/*
 * CompressionStatistics (tree/compression_statistics.cpp): per edge number (breadth-first over a
 * full binary tree of height h: 2^(h+1) - 2 edges) a score per (parent encoding, child encoding).
 * update: score = (max(score, 1) + max(ratio, 1)) / 2.  best: GetBest -- the highest score above 1
 * whose child differs from `to` (and whose parent is `from` when same_beginning); ties go to the
 * smallest (parent, child).  Host-only: these calls do no device work.
 */
gtsc_status gtsc_edge_stats_create(int32_t tree_height, gtsc_edge_stats **out);
gtsc_status gtsc_edge_stats_destroy(gtsc_edge_stats *s);
gtsc_status gtsc_edge_stats_set(gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double value);
gtsc_status gtsc_edge_stats_update(gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double ratio);
gtsc_status gtsc_edge_stats_get(const gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to, double *value);
gtsc_status gtsc_edge_stats_best(const gtsc_edge_stats *s, int32_t edge, int16_t from, int16_t to,
                                 int32_t same_beginning, int16_t *best_from, int16_t *best_to, double *value);
/* every (parent, child) entry of one edge in (parent, child) order: pairs_out 2 per entry */
gtsc_status gtsc_edge_stats_entries(const gtsc_edge_stats *s, int32_t edge, int16_t *pairs_out, double *values_out,
                                    int32_t cap, int32_t *n);
/* CompressionTree::GetEdges (:199-230): edge numbers and pre-order node indices of each edge */
gtsc_status gtsc_tree_edges(const int16_t *nodes, int32_t n_nodes, int32_t *edge_no, int32_t *from_node,
                            int32_t *to_node, int32_t cap, int32_t *n_edges);
/* CompressionTree::UpdateStatistics (:232-240) for a tree with the given node ratios (pre-order) */
gtsc_status gtsc_tree_update_statistics(const int16_t *nodes, const double *ratios, int32_t n_nodes,
                                        gtsc_edge_stats *s);
/*
 * OptimalTree (optimizer/optimal_tree.hpp:24-63): a tree (pre-order nodes + ratios; ratio of the
 * root = the tree's ratio) bound to live statistics `stats`, of which it keeps a snapshot.
 * set_ratio changes one node's ratio (as a compression would); try_correct is TryCorrectTree.
 */
typedef struct gtsc_optimal_tree gtsc_optimal_tree;
gtsc_status gtsc_optimal_tree_create(const int16_t *nodes, const double *ratios, int32_t n_nodes,
                                     gtsc_edge_stats *stats, gtsc_optimal_tree **out);
gtsc_status gtsc_optimal_tree_set_ratio(gtsc_optimal_tree *t, int32_t node, double ratio);
gtsc_status gtsc_optimal_tree_try_correct(gtsc_optimal_tree *t, int32_t *corrected);
gtsc_status gtsc_optimal_tree_get(const gtsc_optimal_tree *t, int16_t *nodes_out, double *ratios_out, int32_t cap,
                                  int32_t *n_nodes);
gtsc_status gtsc_optimal_tree_destroy(gtsc_optimal_tree *t);

/*
 * Delta decode that allocates no device memory (no counterpart in the reference).  For callers that
 * cannot call cudaMalloc -- e.g. code whose device memory is all owned by a host framework's pool.
 * Decodes the delta stream (d_first = the metadata, the column's first value; d_deltas = n_deltas
 * deltas) into d_out, which the caller provides with room for n_deltas + 1 values (16-byte aligned;
 * d_deltas aligned to the element size).  The scan's scratch is a static device array of ~128 KB,
 * reserved on every GPU that loads the library until exit, so at most 2^24 values are decoded per
 * call (GTSC_ERR_CAPACITY beyond).  Each call looks up that array's address on the current device
 * (so a cudaDeviceReset in between is harmless); the first call on a device also loads the library's
 * module there and should come before any stream capture.  Calls share the array: calls whose GPU
 * work overlaps race.
 * Synchronises the stream before returning.
 */
gtsc_status gtsc_delta_decode_noalloc(int32_t dtype, const void *d_first, const void *d_deltas,
                                      uint64_t n_deltas, void *d_out, void *stream);

/*
 * Self-test of the bounded waits (no counterpart in the reference).  Every scan in the library
 * chains its tiles by a decoupled look-back whose waits are bounded: a tile whose predecessor never
 * publishes gives up after a fixed number of polls (about a second), records GTSC_ERR_TIMEOUT in
 * the scan's error word and returns, so a broken predecessor cannot hang the GPU.  This call runs
 * one look-back whose predecessor is never published and returns, in *error_word, what the waiting
 * tile recorded (GTSC_ERR_TIMEOUT when the bound works) and, in *seconds, how long the wait took.
 * The device stays usable afterwards.  Synchronises the stream before returning.
 */
gtsc_status gtsc_selftest_lookback_timeout(int32_t *error_word, double *seconds, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GTSC_H_ */
