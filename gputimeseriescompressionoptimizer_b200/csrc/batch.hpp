// batch.hpp -- the batched multi-column tree engine.
//
// Many columns, each with its own compression tree, are processed together: every tree node is
// split into passes (min/max, histogram, split, pack, ...), passes of the same kind whose inputs
// are ready are grouped into one stage, and a stage is ONE launch whose blocks pull (item, tile)
// work across all columns.  Stream lengths live in device words, so no stage needs the host: a
// whole compress (or decompress) step is a fixed sequence of launches, captured once in a CUDA
// graph and replayed.
#pragma once

#include "common.cuh"
#include "tree.hpp"

namespace gtsc {

// pass kinds (one batched kernel each)
enum BOp : int {
    B_MINMAX = 0,      // min/max accumulators (AFL, scale, patch)
    B_DELTA_ENC,
    B_SCALE_SUB,
    B_AFL_PACK,
    B_HIST,            // dict / const histogram
    B_TOPK,            // one block per item
    B_SPLIT,           // patch / const / dict split (mode in item.mode)
    B_RLE_HEADS,
    B_RLE_LENGTHS,
    B_F2I_STATS,
    B_F2I_ENC,
    B_F2I_RAW,
    B_GFC_COMPRESS,
    B_GFC_SCAN,
    B_GFC_COMPACT,
    B_NONE_COPY,       // decode: none leaf copied to an aligned stream
    // decode
    B_AFL_UNPACK,
    B_DELTA_DEC,
    B_SCALE_ADD,
    B_MERGE,
    B_RLE_SCAN,
    B_RLE_EXPAND,
    B_F2I_DEC,
    B_GFC_SIZES,
    B_GFC_DEC,
    B_VMETA,           // compress: metadata of a node whose output is read through a view
    B_MERGE_COUNT,     // decode: stencil matches per merge tile and per group of 64 tiles
    B_NUM_OPS
};

// Elementwise operations a pass applies to its input stream on the fly (the input "view"), so that
// delta and scale nodes feeding another encoding never write their output: in order,
//   V_DELTA  y[i] = x[i + 1] - x[i]            (one element shorter)
//   V_SCALE  y[i] = x[i] - c                   (c from the scale node's min/max, scale_min)
enum VOp : int8_t { V_NONE = 0, V_DELTA = 1, V_SCALE = 2 };
constexpr int kMaxViewOps = 3;

// A stream: device bytes and their length.  The table lives in device memory; compress passes
// write lengths, the decode parser writes the pointers of streams that sit inside a blob.
struct StreamDesc {
    uint8_t *ptr;
    uint64_t len;   // bytes
    uint64_t cap;   // bytes reserved (arena streams)
    uint64_t pad;
};

// How a decode pass reads one of its inputs.  data >= 0 and afl_meta < 0: the stream `data` (a
// child's decoded stream, or a none leaf inside the blob).  afl_meta >= 0: the child is an AFL
// node whose packed bits are `data` (its none leaf, in the blob) and whose metadata is afl_meta;
// element i is unpacked on the fly.  add[k] >= 0: then add the value in that scale node's metadata
// (a scale child, decoded on the fly).  data < 0: the input comes from in[] as before.
struct DView {
    int32_t data = -1;
    int32_t afl_meta = -1;
    int32_t add[2] = {-1, -1};
};

// One unit of batched work: a pass of one tree node of one column.
struct BItem {
    uint64_t tile_base;          // first global tile of this item
    uint32_t tiles;              // tiles reserved (worst case; tiles past the real length exit)
    int16_t op, mode;            // pass kind; SplitMode / top-k size / merge mode
    int16_t es, order;           // element size, Order of the node's data type
    int32_t dt;
    int32_t in[3];               // input stream ids (-1 = none)
    int32_t out[3];              // output stream ids (compress: meta, out1, out2; decode: out[0])
    uint8_t *scratch;            // the node's scratch: accumulators, look-back state, tables
    uint64_t p[4];               // pass parameters (scratch offsets, capacities)
    int8_t vop[kMaxViewOps];     // the input view: ops applied to in[0] (compress passes)
    int8_t vflags;               // bit 0: AFL width from the view's last scale (no own min/max pass)
    uint8_t *vscr[kMaxViewOps];  // V_SCALE: that scale node's scratch (its MinMaxAcc)
    DView dv[2];                 // decode passes: how in[1] / in[2] are read (see DView)
};

// A tree node as the framing / parse kernels see it.
struct BNodeDev {
    int32_t enc, dt;
    int32_t meta;                // stream id of the node's metadata (-1 for none: 8 size bytes)
    int32_t data;                // none leaves: stream id of the data (-1 otherwise)
    uint64_t meta_dst, data_dst; // destinations in the framed buffer (set by the layout pass)
};
struct BColumnDev {
    int32_t first, n_nodes;      // the column's nodes in the node table, pre-order
};

void launch_frame_sizes(const BColumnDev *cols, int ncols, const BNodeDev *nodes, const StreamDesc *S,
                        unsigned long long *col_off, unsigned long long *total, uint8_t *framed, cudaStream_t s);
void launch_frame_layout(const BColumnDev *cols, int ncols, BNodeDev *nodes, const StreamDesc *S,
                         const unsigned long long *col_off, uint8_t *framed, cudaStream_t s);
void launch_frame_copy(const BItem *items, const uint32_t *item_of, int n_items, uint64_t total_tiles,
                       const BNodeDev *nodes, const StreamDesc *S, uint8_t *framed, cudaStream_t s);
void launch_parse_frames(const BColumnDev *cols, int ncols, const BNodeDev *nodes, StreamDesc *S,
                         unsigned long long *col_off, const uint8_t *const *framed_p,
                         const unsigned long long *framed_bytes_p, uint32_t *status, cudaStream_t s);
void launch_zero_ranges(const unsigned long long *ranges, int n, cudaStream_t s);
uint64_t batch_copy_piece();

struct BatchColumn {
    const void *data;  // device column
    uint64_t bytes;
    int dtype;
};

class BatchEngine;

// Launch parameters chosen per batch by the autotuner (batch_autotune); the defaults are the
// hand-picked values.  Tiles are values per block tile.
struct BatchTuning {
    uint32_t minmax_tile = 8192;   // min/max pass: a multiple of 256 x minmax_vpt, 1K .. 16K
    uint32_t minmax_vpt = 16;      // min/max pass: consecutive values a thread loads per round (1 .. 16)
    uint32_t hist_tile = 32768;    // histogram pass (dict / const), 8K .. 32K
    bool persistent_c = false;     // compress step: one persistent launch instead of the levels
    bool persistent_d = false;     // decompress step: the same
};

// Compile a batch: columns + their (Fix()ed) trees.  Owns the arena and the graphs.
BatchEngine *batch_create(const std::vector<BatchColumn> &cols, const std::vector<Tree> &trees, cudaStream_t s,
                          const BatchTuning &tuning = BatchTuning());
// the batch's launch parameters
BatchTuning batch_tuning(const BatchEngine *e);
// Times candidate launch parameters on the batch's own columns and trees (CUDA events, each
// candidate compiled as a batch of its own): the schedule of each step, then the min/max tile x
// values per thread, then the histogram tile, each kept when it lowers the time of the passes it
// affects.  Returns a batch built with the best parameters (the old one is destroyed), and the
// step times before and after.
struct TuneReport {
    BatchTuning best;
    float ms_default[2] = {0, 0};  // compress, decompress with the default parameters
    float ms_tuned[2] = {0, 0};
    int candidates = 0;
    float seconds = 0;
};
BatchEngine *batch_autotune(BatchEngine *e, cudaStream_t s, TuneReport *report);
void batch_destroy(BatchEngine *e);
// compress all columns into the framed output: uint64 column count, uint64 blob bytes per column,
// then the blobs (CompressionTree::Compress of each column) back to back
void batch_compress(BatchEngine *e, cudaStream_t s);
// new device pointers for the columns (same sizes), used by the next compress
void batch_set_inputs(BatchEngine *e, const std::vector<const void *> &inputs, cudaStream_t s);
// total framed bytes (synchronises) and the device framed buffer
uint64_t batch_output_bytes(BatchEngine *e, cudaStream_t s);
const uint8_t *batch_output(BatchEngine *e);
// per-column blob sizes (synchronises)
std::vector<uint64_t> batch_blob_sizes(BatchEngine *e, cudaStream_t s);
// decompress a framed buffer produced with the same trees (any step) into the columns' outputs
void batch_decompress(BatchEngine *e, const uint8_t *framed, uint64_t framed_bytes,
                      const std::vector<void *> &outputs, cudaStream_t s);
// status word of the last step (0 = ok); synchronises
gtsc_status batch_status(BatchEngine *e, cudaStream_t s);
// number of kernel launches in one compress / decompress step
int batch_launches(BatchEngine *e, bool compress);
// the schedule the steps replay: a launch per (level, pass kind), or one persistent launch per step
// pulling tiles from a device queue (both are captured at creation; the default is the levels)
void batch_set_schedule(BatchEngine *e, bool persistent);
bool batch_schedule(const BatchEngine *e);
// one step run launch by launch with events between launches: per launch its pass kind (a BOp, or
// a negative code for the fixed kernels), its time and the bytes it must move at least
struct BatchLaunchProfile {
    int op;
    float ms;
    uint64_t bytes;
    uint64_t blocks;
};
std::vector<BatchLaunchProfile> batch_profile(BatchEngine *e, bool compress, cudaStream_t s);

// column chunks from host memory through per-group batch engines with overlapped copies
struct Pipeline;
Pipeline *pipeline_create(const std::vector<uint64_t> &bytes, const std::vector<int> &dtypes,
                          const std::vector<Tree> &trees, int groups);
void pipeline_destroy(Pipeline *p);
int pipeline_groups(const Pipeline *p);
const std::vector<int> &pipeline_group_columns(const Pipeline *p, int g);  // ascending column indices
void pipeline_compress_host(Pipeline *p, const void *const *host_cols, uint8_t *host_framed, uint64_t cap,
                            uint64_t *sizes, bool decode);
gtsc_status pipeline_decompress(Pipeline *p);
const void *pipeline_column_input(Pipeline *p, int c);
const void *pipeline_column_output(Pipeline *p, int c);

// ---- the persistent schedule: one launch per step whose blocks pull work from a device queue
//
// The queue is the level schedule laid end to end, in units: the launches in order, each cut into
// units of one tile (look-back passes, taken in the stage launch's claim order: tile j of every
// item before tile j + 1 of any) or of up to kPersistChunk consecutive tiles (the other passes).  A
// unit names its first tile (item, tile) and its tile count; a block claims one unit at a time and
// runs its tiles in order (a chunk walks on into the next item of the same launch), so a look-back
// tile never waits behind other work of the block that holds its predecessor.  An item waits,
// before its first tile, until its column has finished every tile of the earlier levels
// (done[col] >= wait): passes of different columns never depend on one another, and a level only
// follows levels of its own column, so small columns run ahead instead of waiting at every level
// for the largest ones.  Every tile depends only on tiles of lower units (look-back predecessors
// come earlier in claim order, earlier levels earlier in the queue), so the lowest unfinished unit
// can always run and the resident blocks always make progress; each wait is still bounded
// (GTSC_ERR_TIMEOUT).
struct PUnit {
    uint32_t item;        // the item of the unit's first tile (phase item table)
    uint32_t tile_count;  // that tile (low 28 bits) and the unit's tiles (high 4 bits)
};
struct PItem {
    uint32_t col;       // the item's column
    uint32_t wait;      // tiles of that column in earlier levels
};
struct PersistArgs {
    const PUnit *units;
    uint32_t total;     // queue units
    const BItem *items;
    const PItem *pitems;
    uint32_t *done;     // per column: tiles finished (zeroed each step)
    uint32_t *ext;      // per item: 1 + its extent in tiles once a block computed it (zeroed)
    uint32_t *qcounter; // the claim counter (zeroed)
    StreamDesc *S;
    uint32_t *status;
};
constexpr uint32_t kPersistChunk = 8;  // tiles per queue unit of a pass without look-back (<= 15)
// one persistent launch of a whole compress (batch_kernels.cu) or decode (batch_decode.cu) step
void launch_batch_persistent_c(const PersistArgs &a, cudaStream_t s);
void launch_batch_persistent_d(const PersistArgs &a, cudaStream_t s);

// stage launcher (batch_kernels.cu / batch_decode.cu): one launch of `total_tiles` blocks;
// d_item_of[t] = the item (index into d_items) of tile t
void launch_batch_stage(int op, const BItem *d_items, const uint32_t *d_item_of, int n_items, uint64_t total_tiles,
                        StreamDesc *d_streams, uint32_t *d_counter, uint32_t *d_status, cudaStream_t s);

// tile sizes (elements) of the batched passes
constexpr uint32_t kBVPT = 16;         // values per thread of the element-wise and look-back passes
constexpr uint32_t kBTile = 256 * kBVPT; // elements per tile of those passes (256 threads per block)
constexpr uint32_t kBMergeSub = 4;      // kBTile tiles per block of the merge pass
constexpr uint32_t kBGfcChunks = 8;     // GFC chunks (warps) per tile
constexpr uint32_t kBHistSmem = 2048;    // shared hash slots of a histogram block (8-byte values)
constexpr uint32_t kBHistPacked = 4096;  // 8 x this = the bytes of a histogram block's shared table
constexpr uint32_t kBHistSlots16 = 5456; // its slots for values of up to 4 bytes (16-bit counts)
constexpr uint32_t kBHistTileMax = 32768; // largest histogram tile (a 16-bit count holds its values)

// scratch layout of a histogram item
struct BHistHdr {
    unsigned int used;      // slots taken in the global table
    unsigned int special;   // occurrences of the all-ones value
    unsigned int overflow;
    unsigned int pad;       // top-k: blocks finished
};
// header | keys (8 cap) | counts (4 cap) | used slots (4 cap) | NaN lists (32 per tile) | top-k
// partials (96 per tile)
inline uint64_t bhist_bytes(uint64_t cap, uint64_t tiles)
{
    return 16 + 8 * cap + 4 * cap + 4 * cap + 32 * tiles + 96 * tiles + 64;
}

}  // namespace gtsc
